// Individual particles on a lattice: Brownian step, binning by radix sort and
// cell offsets, in-cell A + B -> 0 pairing, compaction.
//
// The reference keeps individuals as 64-bit (cell, id) keys, moves them one
// lattice cell at a time (individual_diffuseX/Y, IndividualSolver.cl:750-1014),
// re-sorts after every move (IndividualSolver::computeDiffusionConstants ->
// sortSpecies, IndividualSolver.cpp:1100-1153, :673-712) and handles births and
// deaths by scans and compaction (maintainPopulation, IndividualSolver.cpp:458-671).
// This path keeps continuous positions (float2) and a species byte per particle;
// a step is
//   move:    x += vx dt + sqrt(2 D dt) z (Box-Muller normals from the particle's
//            Philox stream), reflecting walls, key = floor(y) G + floor(x);
//   bin:     stable radix sort of (key, index) (the move counts the digits, the
//            sort's last pass the particles per cell);
//   react:   in each cell the k-th A (in sorted order) pairs with the k-th B and the
//            pair is removed with probability p (one 32-bit draw per pair against
//            floor(p 2^32));
//   compact: survivors in sorted order.
// React and compact are one kernel over the cells that also scans the counts into
// the cell starts.
// Compiled with -fmad=false: positions must round as the CPU replay does.
#include <cmath>
#include <cstdint>
#include <cuda_runtime.h>
#include "common.cuh"
#include "lookback.cuh"
#include "host_common.h"
#include "sort_kernels.h"
#include "../../include/gpgmp_c.h"

using namespace gpgmp;

namespace {

__device__ __forceinline__ float reflect_into(float x, float L) {
    if (x < 0.0f) x = -x;
    if (x >= L) x = (L + L) - x;
    if (x < 0.0f) x = 0.0f;
    if (x >= L) x = nextafterf(L, 0.0f);
    return x;
}

// The move also counts the radix digits of the new keys for every sort pass (the
// histogram the sort would otherwise read the keys again for).
__global__ void k_move(float* __restrict__ px, float* __restrict__ py, int64_t n, int G, float sig, float ax, float ay,
                       uint32_t seed, uint32_t step, uint32_t* __restrict__ keys, uint32_t* __restrict__ vals,
                       uint32_t* __restrict__ hist, int passes, int rb) {
    __shared__ uint32_t s_h[3 * 1024];   // [passes][1 << rb]: 4 x 256 or up to 3 x 1024
    const int dig = 1 << rb;
    const uint32_t dmask = (uint32_t)dig - 1u;
    for (int i = threadIdx.x; i < passes * dig; i += blockDim.x) s_h[i] = 0;
    __syncthreads();
    const float L = (float)G;
    const int lane = threadIdx.x & 31;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    // whole warps step together (the digit counts below are warp-collective)
    for (int64_t base = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) - lane; base < n; base += stride) {
        const int64_t i = base + lane;
        const bool valid = i < n;
        const unsigned vmask = __ballot_sync(0xffffffffu, valid);
        uint32_t k = 0;
        if (valid) {
            Stream st;
            st.init(seed, 0u, step, (uint32_t)i, PH_PART);
            float z0, z1;
            normal2(st, &z0, &z1);
            float x = px[i] + ax;
            x = x + sig * z0;
            float y = py[i] + ay;
            y = y + sig * z1;
            x = reflect_into(x, L);
            y = reflect_into(y, L);
            px[i] = x;
            py[i] = y;
            k = (uint32_t)(int)y * (uint32_t)G + (uint32_t)(int)x;
            keys[i] = k;
            vals[i] = (uint32_t)i;
        }
        // The particles come in the last step's cell order, so a warp's upper digits
        // are mostly all the same: one add for the warp then, one per lane otherwise.
        const int lead = __ffs(vmask) - 1;
        for (int p = 0; p < passes; ++p) {
            const uint32_t d = (k >> (rb * p)) & dmask;
            const uint32_t d0 = __shfl_sync(0xffffffffu, d, lead);
            if (__all_sync(0xffffffffu, !valid || d == d0)) {
                if (lane == lead) atomicAdd(&s_h[p * dig + d0], (uint32_t)__popc(vmask));
            } else if (valid) {
                atomicAdd(&s_h[p * dig + d], 1u);
            }
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < passes * dig; i += blockDim.x) {
        const uint32_t c = s_h[i];
        if (c) atomicAdd(&hist[i], c);
    }
}

// React and compact in one pass over the cells, with two decoupled look-back scans
// (lookback.cuh).  A tile of 1024 cells (four per thread) takes its cells' starts
// from the scan of the counts; its particles are then one contiguous range of the
// sorted list, whose species bytes the block stages in shared memory.  Each thread
// pairs the A's and B's of its cells there: the k-th A in sorted order with the k-th
// B, a pair going with probability thresh / 2^32 (one 32-bit draw per pair from the
// cell's stream), from species bit masks in a cell of up to 32 particles and by
// walking the staged bytes in a larger one.  Then the tile takes its survivors' output offset from the scan of the
// survivor counts, and each warp writes the survivors of its own threads' cells
// (position and species) with ballot-ranked, coalesced stores: the order of
// compacting the sorted list by alive flags.  The last tile writes the total.  A tile
// with more particles than the staging holds walks each cell in global memory with
// alive flags instead.
constexpr int kRcThreads = 256;
constexpr int kRcCells = 4;
constexpr int kRcTile = kRcThreads * kRcCells;
constexpr int kRcWarps = kRcThreads / 32;
constexpr uint8_t kRcDead = 0xffu;

// exclusive sum over the block (kRcThreads threads); *total = the block's sum
__device__ __forceinline__ uint32_t block_excl_sum(uint32_t v, uint32_t* s_warp, uint32_t* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < kRcWarps ? s_warp[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += t;
        }
        if (lane < kRcWarps) s_warp[lane] = w;
    }
    __syncthreads();
    *total = s_warp[kRcWarps - 1];
    return (warp == 0 ? 0u : s_warp[warp - 1]) + incl - v;
}

// Pairs one cell's A's and B's in order; dead pairs are marked in sp (kRcDead) or,
// with alive != nullptr, cleared in alive.  Returns the number of pairs removed.
template <class SP>
__device__ __forceinline__ uint32_t pair_cell(uint32_t b, uint32_t f, const SP& species, uint32_t seed, uint32_t step,
                                              uint32_t cell, uint32_t thresh, uint8_t* mark, uint32_t* alive) {
    Stream st;
    st.init(seed, 1u, step, cell, PH_PAIR);
    uint32_t ia = b, ib = b, removed = 0;
    for (;;) {
        while (ia < f && species(ia) != 0) ia++;
        while (ib < f && species(ib) != 1) ib++;
        if (ia >= f || ib >= f) break;
        if (st.next() < thresh) {
            if (mark) {
                mark[ia] = kRcDead;
                mark[ib] = kRcDead;
            } else {
                alive[ia] = 0;
                alive[ib] = 0;
            }
            removed++;
        }
        ia++;
        ib++;
    }
    return removed;
}

// scratch (uint64 words): [0] tile counter (u32), error word (u32 at byte 8), total
// (u32 at byte 16), then the status words of the two scans, ntiles each.
// Dynamic shared memory: cap bytes (species of the staged particles).
// (at most 32 registers: eight tiles per SM, so the 1024 tiles of a 1024 x 1024 grid
// are resident in one wave)
__global__ void __launch_bounds__(kRcThreads, 8) k_react_compact(
    const uint32_t* __restrict__ count, uint32_t* __restrict__ start, int64_t ncells,
    const uint32_t* __restrict__ svals, const float* __restrict__ x, const float* __restrict__ y,
    const uint8_t* __restrict__ sp, uint32_t seed, uint32_t step, uint32_t thresh, uint32_t* __restrict__ alive,
    float* __restrict__ x2, float* __restrict__ y2, uint8_t* __restrict__ sp2, uint64_t* __restrict__ scratch,
    uint32_t ntiles, uint32_t cap) {
    extern __shared__ uint8_t s_sp[];          // [cap] species, kRcDead = removed
    __shared__ uint32_t s_tile, s_prefix;
    __shared__ uint32_t s_warp[kRcWarps];
    unsigned int* counter = reinterpret_cast<unsigned int*>(scratch);
    int* err = reinterpret_cast<int*>(scratch) + 2;
    uint32_t* total = reinterpret_cast<uint32_t*>(scratch) + 4;
    uint64_t* status_start = scratch + 4;
    uint64_t* status_out = status_start + ntiles;
    if (threadIdx.x == 0) s_tile = atomicAdd(counter, 1u);
    __syncthreads();
    const uint32_t tile = s_tile;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t c0 = (int64_t)tile * kRcTile + (int64_t)threadIdx.x * kRcCells;
    uint32_t cnt[kRcCells];
    if (c0 + kRcCells <= ncells) {
        const uint4 w = *reinterpret_cast<const uint4*>(count + c0);
        cnt[0] = w.x; cnt[1] = w.y; cnt[2] = w.z; cnt[3] = w.w;
    } else {
#pragma unroll
        for (int j = 0; j < kRcCells; ++j) cnt[j] = c0 + j < ncells ? count[c0 + j] : 0u;
    }
    uint32_t sum = 0;
#pragma unroll
    for (int j = 0; j < kRcCells; ++j) sum += cnt[j];
    uint32_t agg;
    const uint32_t ex = block_excl_sum(sum, s_warp, &agg);
    if (warp == 0) {
        const uint32_t p = warp_lookback_u32(status_start, tile, agg, err);
        if (lane == 0) s_prefix = p;
    }
    __syncthreads();
    const uint32_t S = s_prefix;               // the tile's first particle in the sorted list
    uint32_t o[kRcCells + 1];                  // the cells' offsets within the tile
    o[0] = ex;
#pragma unroll
    for (int j = 0; j < kRcCells; ++j) o[j + 1] = o[j] + cnt[j];
    if (c0 + kRcCells <= ncells) {
        *reinterpret_cast<uint4*>(start + c0) = make_uint4(S + o[0], S + o[1], S + o[2], S + o[3]);
    } else {
#pragma unroll
        for (int j = 0; j < kRcCells; ++j)
            if (c0 + j < ncells) start[c0 + j] = S + o[j];
    }
    const bool staged = agg <= cap;            // the same in every thread of the block
    // the part of the staged range that holds this warp's threads' cells
    const uint32_t w0 = __shfl_sync(0xffffffffu, o[0], 0);
    const uint32_t w1 = __shfl_sync(0xffffffffu, o[kRcCells], 31);
    uint32_t removed = 0;
    if (staged) {
        for (uint32_t p0 = 0; p0 < agg; p0 += 4 * kRcThreads) {
            uint32_t src[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const uint32_t p = p0 + u * kRcThreads + threadIdx.x;
                src[u] = p < agg ? svals[S + p] : 0u;
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const uint32_t p = p0 + u * kRcThreads + threadIdx.x;
                if (p < agg) s_sp[p] = sp[src[u]];
            }
        }
        __syncthreads();
#pragma unroll
        for (int j = 0; j < kRcCells; ++j) {
            if (cnt[j] >= 2) {
                Stream st;
                st.init(seed, 1u, step, (uint32_t)(c0 + j), PH_PAIR);
                if (cnt[j] <= 32) {
                    // species masks of the cell; the k-th set bits of the two masks pair
                    uint32_t am = 0, bm = 0;
                    for (uint32_t q = 0; q < cnt[j]; ++q) {
                        const uint8_t t = s_sp[o[j] + q];
                        am |= (uint32_t)(t == 0) << q;
                        bm |= (uint32_t)(t == 1) << q;
                    }
                    while (am && bm) {
                        const int ia = __ffs(am) - 1, ib = __ffs(bm) - 1;
                        am &= am - 1u;
                        bm &= bm - 1u;
                        if (st.next() < thresh) {
                            s_sp[o[j] + ia] = kRcDead;
                            s_sp[o[j] + ib] = kRcDead;
                            removed++;
                        }
                    }
                } else {
                    uint32_t ia = o[j], ib = o[j];
                    const uint32_t f = o[j + 1];
                    for (;;) {
                        while (ia < f && s_sp[ia] != 0) ia++;
                        while (ib < f && s_sp[ib] != 1) ib++;
                        if (ia >= f || ib >= f) break;
                        if (st.next() < thresh) {
                            s_sp[ia] = kRcDead;
                            s_sp[ib] = kRcDead;
                            removed++;
                        }
                        ia++;
                        ib++;
                    }
                }
            }
        }
    } else {
        const auto global_sp = [&](uint32_t q) { return sp[svals[q]]; };
        for (uint32_t q = S + o[0]; q < S + o[kRcCells]; ++q) alive[q] = 1u;
#pragma unroll
        for (int j = 0; j < kRcCells; ++j) {
            if (cnt[j] >= 2) {
                removed += pair_cell(S + o[j], S + o[j + 1], global_sp, seed, step, (uint32_t)(c0 + j), thresh,
                                     nullptr, alive);
            }
        }
    }
    const uint32_t surv = sum - 2 * removed;
    uint32_t agg2;
    const uint32_t ex2 = block_excl_sum(surv, s_warp, &agg2);
    if (warp == 0) {
        const uint32_t p = warp_lookback_u32(status_out, tile, agg2, err);
        if (lane == 0) {
            s_prefix = p;
            if (tile == ntiles - 1) *total = p + agg2;
        }
    }
    __syncthreads();
    if (staged) {
        // warp w writes the particles of its own threads' cells -- one contiguous part
        // [w0, w1) of the staged range -- in rows of 32; its survivors start where its
        // first lane's exclusive survivor count says
        uint32_t d = s_prefix + __shfl_sync(0xffffffffu, ex2, 0);
        for (uint32_t r = w0; r < w1; r += 32) {
            const uint32_t p = r + lane;
            const bool live = p < w1 && s_sp[p] != kRcDead;
            const unsigned m = __ballot_sync(0xffffffffu, live);
            if (live) {
                const uint32_t dd = d + __popc(m & ((1u << lane) - 1u));
                const uint32_t src = svals[S + p];
                x2[dd] = x[src];
                y2[dd] = y[src];
                sp2[dd] = s_sp[p];
            }
            d += __popc(m);
        }
    } else {
        uint32_t d = s_prefix + ex2;
        for (uint32_t q = S + o[0]; q < S + o[kRcCells]; ++q) {
            if (removed && !alive[q]) continue;
            const uint32_t src = svals[q];
            x2[d] = x[src];
            y2[d] = y[src];
            sp2[d] = sp[src];
            d++;
        }
    }
}

inline unsigned grid_of(int64_t n, int threads) {
    int64_t b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > 148 * 32) b = 148 * 32;
    return (unsigned)b;
}

}  // namespace

struct gpgmp_particles {
    int64_t cap = 0, n = 0;
    int grid = 0;
    float D = 0, vx = 0, vy = 0, dt = 1, p = 0;
    uint32_t seed = 0, thresh = 0;
    int32_t step = 0;
    int key_bits = 32;
    cudaStream_t stream = nullptr;
    float *x = nullptr, *y = nullptr, *x2 = nullptr, *y2 = nullptr;
    uint8_t *sp = nullptr, *sp2 = nullptr;
    uint32_t *keys = nullptr, *vals = nullptr, *skeys = nullptr, *svals = nullptr;
    uint32_t *start = nullptr, *count = nullptr, *alive = nullptr;
    void* sort_scratch = nullptr;
    uint64_t* rc_scratch = nullptr;  // react + compact: tile counter, error word, total, scan status words
    uint32_t rc_tiles = 0;
    uint32_t* host_tail = nullptr;   // pinned: the number of particles after a step
};

#define CK(expr)                                                                                              \
    do {                                                                                                      \
        cudaError_t e_ = (expr);                                                                              \
        if (e_ != cudaSuccess) return set_error(GPGMP_ERR_CUDA, "%s: %s", #expr, cudaGetErrorString(e_));    \
    } while (0)

extern "C" {

int gpgmp_particles_destroy(gpgmp_particles* h) {
    if (!h) return GPGMP_OK;
    cudaStreamSynchronize(h->stream);
    void* ptrs[] = {h->x, h->y, h->x2, h->y2, h->sp, h->sp2, h->keys, h->vals, h->skeys, h->svals, h->start,
                    h->count, h->alive, h->sort_scratch, h->rc_scratch};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (h->host_tail) cudaFreeHost(h->host_tail);
    delete h;
    return GPGMP_OK;
}

int gpgmp_particles_create(int64_t capacity, int32_t grid, float D, float vx, float vy, float dt, float p_react,
                           uint32_t seed, gpgmp_particles** out) {
    if (!out || capacity <= 0 || capacity >= ((int64_t)1 << 30) || grid <= 0 || grid > 32768 || !(dt > 0) ||
        !(D >= 0) || !(p_react >= 0) || !(p_react <= 1))
        return set_error(GPGMP_ERR_INVALID, "bad particle system parameters");
    auto* h = new gpgmp_particles();
    h->cap = capacity;
    h->grid = grid;
    h->D = D; h->vx = vx; h->vy = vy; h->dt = dt; h->p = p_react;
    h->seed = seed;
    h->thresh = (uint32_t)std::floor((double)p_react * 4294967296.0 < 4294967295.0
                                         ? (double)p_react * 4294967296.0 : 4294967295.0);
    const int64_t ncells = (int64_t)grid * grid;
    int bits = 1;
    while (((int64_t)1 << bits) < ncells) ++bits;
    h->key_bits = bits;
    const size_t n4 = sizeof(uint32_t) * (size_t)capacity;
    cudaError_t e = cudaSuccess;
    auto A = [&](void** p, size_t b) { if (e == cudaSuccess) e = cudaMalloc(p, b); };
    A((void**)&h->x, sizeof(float) * capacity); A((void**)&h->y, sizeof(float) * capacity);
    A((void**)&h->x2, sizeof(float) * capacity); A((void**)&h->y2, sizeof(float) * capacity);
    A((void**)&h->sp, capacity); A((void**)&h->sp2, capacity);
    A((void**)&h->keys, n4); A((void**)&h->vals, n4); A((void**)&h->skeys, n4); A((void**)&h->svals, n4);
    A((void**)&h->alive, n4);
    A((void**)&h->start, sizeof(uint32_t) * (size_t)ncells); A((void**)&h->count, sizeof(uint32_t) * (size_t)ncells);
    A(&h->sort_scratch, sort_layout(capacity, bits).bytes);
    h->rc_tiles = (uint32_t)((ncells + kRcTile - 1) / kRcTile);
    A((void**)&h->rc_scratch, sizeof(uint64_t) * (4 + 2 * (size_t)h->rc_tiles));
    if (e == cudaSuccess) e = cudaMallocHost((void**)&h->host_tail, 2 * sizeof(uint32_t));
    if (e != cudaSuccess) {
        int c = set_error(e == cudaErrorMemoryAllocation ? GPGMP_ERR_NOMEM : GPGMP_ERR_CUDA, "allocation: %s",
                          cudaGetErrorString(e));
        gpgmp_particles_destroy(h);
        return c;
    }
    *out = h;
    return GPGMP_OK;
}

int gpgmp_particles_set_stream(gpgmp_particles* h, void* stream) {
    if (!h) return set_error(GPGMP_ERR_INVALID, "handle is NULL");
    h->stream = (cudaStream_t)stream;
    return GPGMP_OK;
}

int gpgmp_particles_set(gpgmp_particles* h, const float* x, const float* y, const uint8_t* species, int64_t n,
                        int32_t step) {
    if (!h || n < 0 || n > h->cap || (n > 0 && (!x || !y || !species))) return set_error(GPGMP_ERR_INVALID, "bad argument");
    CK(cudaMemcpyAsync(h->x, x, sizeof(float) * n, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->y, y, sizeof(float) * n, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->sp, species, n, cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    h->n = n;
    h->step = step;
    return GPGMP_OK;
}

int gpgmp_particles_get(gpgmp_particles* h, float* x, float* y, uint8_t* species, int64_t* n) {
    if (!h || !n) return set_error(GPGMP_ERR_INVALID, "bad argument");
    if (x) CK(cudaMemcpyAsync(x, h->x, sizeof(float) * h->n, cudaMemcpyDeviceToHost, h->stream));
    if (y) CK(cudaMemcpyAsync(y, h->y, sizeof(float) * h->n, cudaMemcpyDeviceToHost, h->stream));
    if (species) CK(cudaMemcpyAsync(species, h->sp, h->n, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    *n = h->n;
    return GPGMP_OK;
}

// One step; n of the next step is read back (4 + 4 bytes) at its end.
static int particles_step_one(gpgmp_particles* h) {
    cudaStream_t st = h->stream;
    const int64_t n = h->n;
    const int64_t ncells = (int64_t)h->grid * h->grid;
    const float sig = sqrtf(2.0f * h->D * h->dt);
    const float ax = h->vx * h->dt, ay = h->vy * h->dt;
    const uint32_t step = (uint32_t)h->step;
    CK(cudaMemsetAsync(h->count, 0, sizeof(uint32_t) * (size_t)ncells, st));
    if (n > 0) {
        CK(radix_sort_begin(n, h->key_bits, h->sort_scratch, st));
        const SortLayout L = sort_layout(n, h->key_bits);
        k_move<<<grid_of(n, 256 * 8), 256, 0, st>>>(h->x, h->y, n, h->grid, sig, ax, ay, h->seed, step, h->keys,
                                                     h->vals, radix_sort_hist(n, h->key_bits, h->sort_scratch),
                                                     L.passes, L.digit_bits);
        CK(cudaGetLastError());
        // the last pass also counts the particles per cell
        CK(radix_sort_finish(h->keys, h->vals, h->skeys, h->svals, n, h->key_bits, h->sort_scratch, st, h->count,
                             ncells));
    }
    CK(cudaMemsetAsync(h->rc_scratch, 0, sizeof(uint64_t) * (4 + 2 * (size_t)h->rc_tiles), st));
    // staging for twice the mean number of particles per tile (+ 1024), up to 47 KB
    // (with the static shared memory, within the 48 KB a launch gets without opting in)
    uint64_t want = (uint64_t)(2.0 * (double)n * kRcTile / (double)ncells) + 1024;
    if (want > 47 * 1024) want = 47 * 1024;
    const uint32_t cap = (uint32_t)want;
    k_react_compact<<<h->rc_tiles, kRcThreads, cap, st>>>(
        h->count, h->start, ncells, h->svals, h->x, h->y, h->sp, h->seed, step, h->thresh, h->alive, h->x2, h->y2,
        h->sp2, h->rc_scratch, h->rc_tiles, cap);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(&h->host_tail[0], reinterpret_cast<uint32_t*>(h->rc_scratch) + 4, sizeof(uint32_t),
                       cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    h->n = (int64_t)h->host_tail[0];
    {
        float* t;
        t = h->x; h->x = h->x2; h->x2 = t;
        t = h->y; h->y = h->y2; h->y2 = t;
        uint8_t* ts = h->sp; h->sp = h->sp2; h->sp2 = ts;
    }
    h->step++;
    return GPGMP_OK;
}

int gpgmp_particles_step(gpgmp_particles* h, int32_t nsteps) {
    if (!h || nsteps < 0) return set_error(GPGMP_ERR_INVALID, "bad argument");
    for (int s = 0; s < nsteps; ++s) {
        int rc = particles_step_one(h);
        if (rc) return rc;
    }
    return GPGMP_OK;
}

// start/count of the last step's binning (before the reaction removed pairs), the
// sorted keys and the index permutation of that step
int gpgmp_particles_bins(gpgmp_particles* h, uint32_t* start, uint32_t* count, uint32_t* sorted_keys,
                         uint32_t* sorted_index, int64_t* n_binned) {
    if (!h) return set_error(GPGMP_ERR_INVALID, "handle is NULL");
    const int64_t ncells = (int64_t)h->grid * h->grid;
    if (start) CK(cudaMemcpyAsync(start, h->start, sizeof(uint32_t) * ncells, cudaMemcpyDeviceToHost, h->stream));
    if (count) CK(cudaMemcpyAsync(count, h->count, sizeof(uint32_t) * ncells, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    int64_t nb = 0;
    if (count) for (int64_t c = 0; c < ncells; ++c) nb += count[c];
    if (sorted_keys && nb) CK(cudaMemcpy(sorted_keys, h->skeys, sizeof(uint32_t) * nb, cudaMemcpyDeviceToHost));
    if (sorted_index && nb) CK(cudaMemcpy(sorted_index, h->svals, sizeof(uint32_t) * nb, cudaMemcpyDeviceToHost));
    if (n_binned) *n_binned = nb;
    return GPGMP_OK;
}

int gpgmp_particles_status(gpgmp_particles* h, int32_t* status) {
    if (!h || !status) return set_error(GPGMP_ERR_INVALID, "bad argument");
    const SortLayout L = sort_layout(h->cap, h->key_bits);
    int a = 0, b = 0;
    CK(cudaMemcpy(&a, (const char*)h->sort_scratch + L.off_counters + 16, sizeof(int), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(&b, (const char*)h->rc_scratch + 8, sizeof(int), cudaMemcpyDeviceToHost));
    *status = (a || b) ? GPGMP_ERR_TIMEOUT : GPGMP_OK;
    return GPGMP_OK;
}

}  // extern "C"
