// Individual-particle population bookkeeping: after a reaction window changed the
// per-cell counts, bring the cell-sorted list of individuals back in line with them.
//
// The reference does this with maintainPopulation, a segmented scan over the grid,
// reduction offsets over the particle list, scatter / new-particle / lost-particle
// kernels and a final copy (IndividualSolver.cpp:458-671, IndividualSolver.cl:
// 1017-1882, doc/source/individual.rst).  Here two kernels do it:
//   1. k_pop_plan, one pass over the cells: is = current count, goal = target count,
//      births = goal - is, kills = is - goal (each clamped at 0), and the exclusive
//      scans of goal, births and kills in one single-pass decoupled look-back
//      (lookback.cuh): the new cell starts, the cell's first id in the old pool and
//      the cell's first slot in the new pool.  A cell of at most 32 individuals that
//      loses some chooses them here, uniformly without replacement (selection
//      sampling, one Philox draw per candidate while removals remain), as a bit mask.
//      The last tile writes the totals.
//   2. k_pop_move, three independent parts, each writing its own outputs:
//      - every individual of a cell with a mask (or that loses nobody) goes to the
//        new list at new start + births + (its rank among the cell's survivors), or,
//        if removed, to the new pool at the cell's first slot + (its rank among the
//        removed);
//      - a cell that gains takes its new ids from the old pool at birth_off[c] and
//        puts them first in the cell; a larger cell that loses chooses its removals
//        the same way as the plan, one candidate after another;
//      - the unused rest of the old pool follows the removed ids in the new pool.
//   The move kernel first checks the totals against the output capacities and the
//   look-back error word, and writes nothing when a check fails.  The host reads the
//   totals and the check words back once, after both kernels.
// Because the new list is laid out by a scan over the cells, no segmented scan is
// needed: a cell that was empty and a cell that was occupied are placed the same way.
#include <atomic>
#include <cstdio>
#include <cstring>
#include "common.cuh"
#include "host_common.h"
#include "lookback.cuh"
#include "sort_kernels.h"
#include "../../include/gpgmp_c.h"

namespace gpgmp {
namespace {

constexpr int kPlanThreads = 512;
constexpr int kPlanItems = 8;
constexpr int kPlanTile = kPlanThreads * kPlanItems;   // 4096 cells
constexpr int kMoveThreads = 256;
constexpr int kMoveUnroll = 4;   // independent loads in flight per thread
constexpr uint32_t kMaskCell = 32;     // cells of at most this many individuals get a removal mask
constexpr uint32_t kHeavy = 1u << 31;  // CellPlan::kill_off flag: removals chosen in the move kernel

// check codes written by k_pop_move
constexpr int kPopShortPool = 1, kPopListFull = 2, kPopPoolFull = 3;

// head of the scratch, cleared before every call
struct PopHeader {
    uint32_t tile_counter;
    int32_t lookback_err;
    int32_t check;
    uint32_t pad0;
    unsigned long long goal_total;   // 64-bit sum of the goals (cannot wrap)
    uint32_t totals[3];              // goal, births, kills, as the 32-bit scans see them
    uint32_t pad1;
    uint64_t pad2[3];
};
static_assert(sizeof(PopHeader) == 64, "header size");

// one thread's pinned landing place for the 64-byte header readback
struct PinnedHeader {
    PopHeader* p = nullptr;
    ~PinnedHeader() {
        if (p) cudaFreeHost(p);
    }
};

// what the move kernel needs about one cell, in one 16-byte load
struct __align__(16) CellPlan {
    uint32_t surv_base;   // new position of the cell's first survivor: new start + births
    uint32_t start;       // old start of the cell
    uint32_t mask;        // removal mask of a cell of at most kMaskCell individuals (bit r: r-th removed)
    uint32_t kill_off;    // first slot of the cell's removed ids in the new pool; | kHeavy
};

// Selection sampling (Knuth, TAOCP vol. 2, 3.4.2 algorithm S) of kills among is
// candidates: candidate i is removed with probability krem / (is - i); draws stop
// once every removal is chosen.  The stream is keyed by (seed, step, cell).
struct Selector {
    Stream st;
    uint32_t is, krem, i;
    __device__ __forceinline__ Selector(uint32_t seed, uint32_t step, uint32_t cell, uint32_t is_, uint32_t kills)
        : is(is_), krem(kills), i(0) {
        st.init(seed, 0u, step, cell, PH_POP);
    }
    // fate of the next candidate: removed iff u (is - i) < krem for u = x / 2^32, x the
    // draw, evaluated exactly in 64-bit integers
    __device__ __forceinline__ bool removed() {
        bool r = false;
        if (krem > 0) {
            const uint32_t x = st.next();
            r = (uint64_t)(is - i) * x < ((uint64_t)krem << 32);
            krem -= r ? 1u : 0u;
        }
        ++i;
        return r;
    }
};

// Removal masks of a warp's listed cells, one cell per lane at a time; cell of list
// entry e is base + (e & 255).
__device__ __forceinline__ void warp_masks(const uint32_t* list, uint32_t* mask, uint32_t nlist, uint32_t seed,
                                           uint32_t step, int64_t base) {
    for (uint32_t j = threadIdx.x & 31; j < nlist; j += 32) {
        const uint32_t e = list[j], local = e & 255u, is = (e >> 8) & 255u, kills = e >> 16;
        Selector sel(seed, step, (uint32_t)(base + local), is, kills);
        uint32_t m = 0u;
        for (uint32_t r = 0; r < is && sel.krem > 0; ++r)
            if (sel.removed()) m |= 1u << r;
        mask[local] = m;
    }
    __syncwarp();
}

// Cells are read and written warp-striped (item q of lane l of warp w is cell
// tile_base + 256 w + 32 q + l for 8 items), so every access is one coalesced 128-byte row; the
// scans run in that order: a warp scan per item row, carried across the rows.
__global__ void __launch_bounds__(kPlanThreads, 2)
    k_pop_plan(const uint32_t* __restrict__ start, const uint32_t* __restrict__ count,
               const int32_t* __restrict__ goal, int64_t ncells, uint32_t seed, uint32_t step,
               uint32_t* __restrict__ new_start, uint32_t* __restrict__ birth_off, CellPlan* __restrict__ plan,
               PopHeader* __restrict__ head, uint64_t* __restrict__ status, int64_t tiles) {
    __shared__ uint32_t s_tile;
    __shared__ uint32_t s_warp[3][kPlanThreads / 32];
    __shared__ uint32_t s_prefix[3];
    __shared__ uint32_t s_list[kPlanThreads / 32][32 * kPlanItems];   // per warp: its cells that need a mask
    __shared__ uint32_t s_mask[kPlanThreads / 32][32 * kPlanItems];
    if (threadIdx.x == 0) s_tile = atomicAdd(&head->tile_counter, 1u);
    __syncthreads();
    const uint32_t tile = s_tile;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t seg = (int64_t)tile * kPlanTile + (int64_t)warp * (32 * kPlanItems) + lane;
    uint32_t is[kPlanItems], g[kPlanItems], ex[3][kPlanItems];
    uint32_t run[3] = {0u, 0u, 0u};
    unsigned long long gsum = 0;
#pragma unroll
    for (int q = 0; q < kPlanItems; ++q) {
        const int64_t c = seg + 32 * q;
        is[q] = 0u;
        g[q] = 0u;
        if (c < ncells) {
            is[q] = __ldg(count + c);
            const int32_t g0 = __ldg(goal + c);
            g[q] = g0 > 0 ? (uint32_t)g0 : 0u;
        }
    }
#pragma unroll
    for (int q = 0; q < kPlanItems; ++q) {
        const uint32_t v[3] = {g[q], g[q] > is[q] ? g[q] - is[q] : 0u, is[q] > g[q] ? is[q] - g[q] : 0u};
        gsum += g[q];
#pragma unroll
        for (int ch = 0; ch < 3; ++ch) {
            uint32_t x = v[ch];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t t = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o) x += t;
            }
            ex[ch][q] = run[ch] + x - v[ch];
            run[ch] += __shfl_sync(0xffffffffu, x, 31);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) gsum += __shfl_xor_sync(0xffffffffu, gsum, o);
    if (lane == 0) {
        if (gsum) atomicAdd(&head->goal_total, gsum);
        s_warp[0][warp] = run[0];
        s_warp[1][warp] = run[1];
        s_warp[2][warp] = run[2];
    }
    // the warp's cells that need a removal mask, compacted so that every lane draws
    // for one of them at a time (local index 32 q + lane | is << 8 | kills << 16)
    uint32_t nlist = 0;
#pragma unroll
    for (int q = 0; q < kPlanItems; ++q) {
        const bool m = is[q] > g[q] && is[q] <= kMaskCell;
        const unsigned bal = __ballot_sync(0xffffffffu, m);
        if (m)
            s_list[warp][nlist + __popc(bal & ((1u << lane) - 1u))] =
                (uint32_t)(32 * q + lane) | (is[q] << 8) | ((is[q] - g[q]) << 16);
        nlist += __popc(bal);
    }
    __syncwarp();
    __syncthreads();
    // warps 0-2 look back first (the other tiles wait for them); the rest draw first
    if (warp >= 3) warp_masks(s_list[warp], s_mask[warp], nlist, seed, step, seg - lane);
    if (warp < 3) {   // warp ch scans the warp totals of channel ch, then looks back for it
        const int ch = warp;
        uint32_t w = lane < kPlanThreads / 32 ? s_warp[ch][lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += t;
        }
        const uint32_t aggregate = __shfl_sync(0xffffffffu, w, kPlanThreads / 32 - 1);
        const uint32_t wexcl = w - (lane < kPlanThreads / 32 ? s_warp[ch][lane] : 0u);
        __syncwarp();
        if (lane < kPlanThreads / 32) s_warp[ch][lane] = wexcl;   // exclusive over warps
        const uint32_t exclusive =
            warp_lookback_u32(status + (size_t)ch * tiles, tile, aggregate, &head->lookback_err);
        if (lane == 0) {
            s_prefix[ch] = exclusive;
            if ((int64_t)tile == tiles - 1) head->totals[ch] = exclusive + aggregate;
        }
        warp_masks(s_list[warp], s_mask[warp], nlist, seed, step, seg - lane);
    }
    __syncthreads();
    uint32_t off[3];
#pragma unroll
    for (int ch = 0; ch < 3; ++ch) off[ch] = s_prefix[ch] + s_warp[ch][warp];
#pragma unroll
    for (int q = 0; q < kPlanItems; ++q) {
        const int64_t c = seg + 32 * q;
        if (c >= ncells) continue;
        const uint32_t ns = off[0] + ex[0][q], bo = off[1] + ex[1][q], ko = off[2] + ex[2][q];
        CellPlan p;
        p.surv_base = ns + (g[q] > is[q] ? g[q] - is[q] : 0u);
        p.start = __ldg(start + c);
        p.mask = 0u;
        p.kill_off = ko;
        if (is[q] > g[q]) {
            if (is[q] <= kMaskCell) p.mask = s_mask[warp][32 * q + lane];
            else p.kill_off |= kHeavy;
        }
        new_start[c] = ns;
        birth_off[c] = bo;
        plan[c] = p;
    }
}

__device__ __forceinline__ void move_one(uint32_t c, uint32_t id, int64_t i, const CellPlan& p,
                                         uint32_t* __restrict__ keys_out, uint32_t* __restrict__ ids_out,
                                         uint32_t* __restrict__ pool_out) {
    if (p.kill_off & kHeavy) return;
    const uint32_t r = (uint32_t)(i - p.start);
    uint32_t o = p.surv_base + r;
    if (p.mask) {   // the cell holds at most kMaskCell individuals, so r < 32
        const uint32_t before = __popc(p.mask & ((1u << r) - 1u));
        if ((p.mask >> r) & 1u) {
            pool_out[p.kill_off + before] = id;
            return;
        }
        o -= before;
    }
    keys_out[o] = c;
    ids_out[o] = id;
}

__global__ void __launch_bounds__(kMoveThreads, 6)
    k_pop_move(const uint32_t* __restrict__ keys, const uint32_t* __restrict__ ids, int64_t n,
               const uint32_t* __restrict__ count, const int32_t* __restrict__ goal, int64_t ncells,
               const uint32_t* __restrict__ pool, int64_t n_pool, uint32_t seed, uint32_t step,
               const uint32_t* __restrict__ new_start, const uint32_t* __restrict__ birth_off,
               const CellPlan* __restrict__ plan, uint32_t* __restrict__ keys_out, uint32_t* __restrict__ ids_out,
               int64_t capacity_out, uint32_t* __restrict__ pool_out, int64_t pool_capacity,
               PopHeader* __restrict__ head) {
    if (head->lookback_err) return;
    const int64_t B = head->totals[1], K = head->totals[2];
    int check = 0;
    if (B > n_pool) check = kPopShortPool;
    else if ((int64_t)head->goal_total > capacity_out) check = kPopListFull;
    else if (n_pool - B + K > pool_capacity) check = kPopPoolFull;
    if (check) {
        if (blockIdx.x == 0 && threadIdx.x == 0) head->check = check;
        return;
    }
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t t0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    // every individual of a cell whose removals are in its mask (or that loses nobody),
    // kMoveUnroll at a time so that their loads are in flight together
    int64_t i = t0;
    for (; i + (kMoveUnroll - 1) * stride < n; i += kMoveUnroll * stride) {
        uint32_t c[kMoveUnroll], id[kMoveUnroll];
        CellPlan p[kMoveUnroll];
#pragma unroll
        for (int u = 0; u < kMoveUnroll; ++u) {
            c[u] = keys[i + u * stride];
            id[u] = ids[i + u * stride];
        }
#pragma unroll
        for (int u = 0; u < kMoveUnroll; ++u) {
            if ((int64_t)c[u] < ncells) p[u] = plan[c[u]];
            else p[u].kill_off = kHeavy;
        }
#pragma unroll
        for (int u = 0; u < kMoveUnroll; ++u) move_one(c[u], id[u], i + u * stride, p[u], keys_out, ids_out, pool_out);
    }
    for (; i < n; i += stride) {
        const uint32_t c = keys[i];
        if ((int64_t)c >= ncells) continue;
        move_one(c, ids[i], i, plan[c], keys_out, ids_out, pool_out);
    }
    // cells that gain, and cells too large for a mask that lose; the counts of
    // kMoveUnroll cells are loaded together
    for (int64_t c0 = t0; c0 < ncells; c0 += kMoveUnroll * stride) {
        uint32_t is[kMoveUnroll], g[kMoveUnroll];
#pragma unroll
        for (int u = 0; u < kMoveUnroll; ++u) {
            const int64_t c = c0 + u * stride;
            is[u] = 0u;
            g[u] = 0u;
            if (c < ncells) {
                is[u] = count[c];
                const int32_t g0 = goal[c];
                g[u] = g0 > 0 ? (uint32_t)g0 : 0u;
            }
        }
#pragma unroll
        for (int u = 0; u < kMoveUnroll; ++u) {
            const int64_t c = c0 + u * stride;
            if (g[u] > is[u]) {
                const uint32_t o = new_start[c], p = birth_off[c];
                for (uint32_t j = 0; j < g[u] - is[u]; ++j) {
                    keys_out[o + j] = (uint32_t)c;
                    ids_out[o + j] = pool[p + j];
                }
            } else if (is[u] > kMaskCell && is[u] > g[u]) {
                const CellPlan pl = plan[c];
                Selector sel(seed, step, (uint32_t)c, is[u], is[u] - g[u]);
                uint32_t o = pl.surv_base, ko = pl.kill_off & ~kHeavy;
                for (uint32_t r = 0; r < is[u]; ++r) {
                    const uint32_t id = ids[pl.start + r];
                    if (sel.removed()) {
                        pool_out[ko++] = id;
                    } else {
                        keys_out[o] = (uint32_t)c;
                        ids_out[o++] = id;
                    }
                }
            }
        }
    }
    // the unused rest of the old pool, after the removed ids
    const int64_t rest = n_pool - B;
    int64_t t = t0;
    for (; t + (kMoveUnroll - 1) * stride < rest; t += kMoveUnroll * stride) {
        uint32_t v[kMoveUnroll];
#pragma unroll
        for (int u = 0; u < kMoveUnroll; ++u) v[u] = pool[B + t + u * stride];
#pragma unroll
        for (int u = 0; u < kMoveUnroll; ++u) pool_out[K + t + u * stride] = v[u];
    }
    for (; t < rest; t += stride) pool_out[K + t] = pool[B + t];
}

struct PopLayout {
    int64_t tiles;
    size_t head, status, new_start, birth_off, plan, bytes;
};

size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

PopLayout pop_layout(int64_t ncells) {
    PopLayout L;
    L.tiles = (ncells + kPlanTile - 1) / kPlanTile;
    size_t o = 0;
    const size_t nc = (size_t)ncells;
    L.head = o; o = align256(o + sizeof(PopHeader));
    L.status = o; o = align256(o + 3 * sizeof(uint64_t) * (size_t)L.tiles);
    L.new_start = o; o = align256(o + 4 * nc);
    L.birth_off = o; o = align256(o + 4 * nc);
    L.plan = o; o = align256(o + sizeof(CellPlan) * nc);
    L.bytes = o;
    return L;
}

// one wave of the move kernel: the blocks that fit on the device at once (looked up
// once per device), fewer for small work
unsigned move_grid(int64_t work) {
    static std::atomic<int> resident[64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) dev = -1;
    int wave = 148 * 6;
    if (dev >= 0) {
        if (!resident[dev].load()) {
            int sms = 0, per_sm = 0;
            if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess &&
                cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pop_move, kMoveThreads, 0) == cudaSuccess &&
                sms > 0 && per_sm > 0)
                resident[dev] = sms * per_sm;
            else
                resident[dev] = wave;
        }
        wave = resident[dev].load();
    }
    int64_t b = (work + kMoveThreads - 1) / kMoveThreads;
    if (b < 1) b = 1;
    if (b > wave) b = wave;
    return (unsigned)b;
}

#define CK(expr)                                                                                           \
    do {                                                                                                   \
        cudaError_t e_ = (expr);                                                                           \
        if (e_ != cudaSuccess) return set_error(GPGMP_ERR_CUDA, "%s: %s", #expr, cudaGetErrorString(e_)); \
    } while (0)

}  // namespace
}  // namespace gpgmp

using namespace gpgmp;

extern "C" {

int gpgmp_population_scratch_bytes(int64_t n_active, int64_t ncells, size_t* bytes) {
    if (!bytes || n_active < 0 || ncells <= 0) return set_error(GPGMP_ERR_INVALID, "bad argument");
    *bytes = pop_layout(ncells).bytes;
    return GPGMP_OK;
}

int gpgmp_population_maintain(const uint32_t* keys, const uint32_t* ids, int64_t n_active, const uint32_t* cell_start,
                              const uint32_t* cell_count, const int32_t* goal, int64_t ncells, const uint32_t* pool,
                              int64_t n_pool, uint32_t seed, uint32_t step, uint32_t* keys_out, uint32_t* ids_out,
                              int64_t capacity_out, uint32_t* pool_out, int64_t pool_capacity, uint32_t* start_out,
                              int64_t* n_active_out, int64_t* n_pool_out, void* scratch, size_t scratch_bytes,
                              void* stream) {
    return gpgmp::population_maintain(keys, ids, n_active, cell_start, cell_count, goal, ncells, pool, n_pool, seed,
                                      step, keys_out, ids_out, capacity_out, pool_out, pool_capacity, start_out,
                                      n_active_out, n_pool_out, nullptr, scratch, scratch_bytes, stream);
}

}  // extern "C"

namespace gpgmp {

int population_maintain(const uint32_t* keys, const uint32_t* ids, int64_t n_active, const uint32_t* cell_start,
                        const uint32_t* cell_count, const int32_t* goal, int64_t ncells, const uint32_t* pool,
                        int64_t n_pool, uint32_t seed, uint32_t step, uint32_t* keys_out, uint32_t* ids_out,
                        int64_t capacity_out, uint32_t* pool_out, int64_t pool_capacity, uint32_t* start_out,
                        int64_t* n_active_out, int64_t* n_pool_out, int64_t* births_out, void* scratch,
                        size_t scratch_bytes, void* stream) {
    if (n_active < 0 || n_pool < 0 || ncells <= 0 || n_active >= ((int64_t)1 << 31) || ncells >= ((int64_t)1 << 31) ||
        n_pool >= ((int64_t)1 << 31))
        return set_error(GPGMP_ERR_INVALID, "bad sizes");
    if (!cell_start || !cell_count || !goal || !keys_out || !ids_out || !pool_out || !n_active_out || !n_pool_out ||
        !scratch || (n_active > 0 && (!keys || !ids)) || (n_pool > 0 && !pool))
        return set_error(GPGMP_ERR_INVALID, "NULL argument");
    const PopLayout L = pop_layout(ncells);
    if (scratch_bytes < L.bytes) return set_error(GPGMP_ERR_INVALID, "scratch too small");
    // list positions are 32-bit: what the kernels may write stays below 2^31
    const int64_t kMax32 = ((int64_t)1 << 31) - 1;
    const int64_t cap_out = capacity_out < kMax32 ? capacity_out : kMax32;
    const int64_t cap_pool = pool_capacity < kMax32 ? pool_capacity : kMax32;
    cudaStream_t st = (cudaStream_t)stream;
    char* base = (char*)scratch;
    PopHeader* head = (PopHeader*)(base + L.head);
    uint64_t* status = (uint64_t*)(base + L.status);
    uint32_t* new_start = start_out ? start_out : (uint32_t*)(base + L.new_start);
    uint32_t* birth_off = (uint32_t*)(base + L.birth_off);
    CellPlan* plan = (CellPlan*)(base + L.plan);
    CK(cudaMemsetAsync(base, 0, L.status + 3 * sizeof(uint64_t) * (size_t)L.tiles, st));
    k_pop_plan<<<(unsigned)L.tiles, kPlanThreads, 0, st>>>(cell_start, cell_count, goal, ncells, seed, step, new_start,
                                                            birth_off, plan, head, status, L.tiles);
    CK(cudaGetLastError());
    int64_t work = n_active > ncells ? n_active : ncells;
    if (n_pool > work) work = n_pool;
    k_pop_move<<<move_grid(work), kMoveThreads, 0, st>>>(keys, ids, n_active, cell_count, goal, ncells, pool, n_pool,
                                                         seed, step, new_start, birth_off, plan, keys_out, ids_out,
                                                         cap_out, pool_out, cap_pool, head);
    CK(cudaGetLastError());
    // the header comes back into this thread's pinned copy (a plain async copy, no
    // staging through a pageable buffer); a call returns only after its copy landed
    thread_local PinnedHeader t_pinned;
    if (!t_pinned.p && cudaMallocHost((void**)&t_pinned.p, sizeof(PopHeader)) != cudaSuccess) {
        cudaGetLastError();
        t_pinned.p = nullptr;
    }
    PopHeader h_stack;
    PopHeader* hp = t_pinned.p ? t_pinned.p : &h_stack;
    CK(cudaMemcpyAsync(hp, head, sizeof(PopHeader), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    const PopHeader h = *hp;
    if (h.lookback_err) return set_error(GPGMP_ERR_TIMEOUT, "a scan's look-back wait gave up");
    const int64_t n_new = (int64_t)h.goal_total, B = h.totals[1], K = h.totals[2];
    if (h.check == kPopShortPool)
        return set_error(GPGMP_ERR_INVALID, "%lld new individuals but only %lld free ids", (long long)B,
                         (long long)n_pool);
    if (h.check == kPopListFull)
        return set_error(GPGMP_ERR_INVALID, "output list holds %lld of %lld individuals", (long long)cap_out,
                         (long long)n_new);
    if (h.check == kPopPoolFull)
        return set_error(GPGMP_ERR_INVALID, "output pool holds %lld of %lld ids", (long long)cap_pool,
                         (long long)(n_pool - B + K));
    *n_active_out = n_new;
    *n_pool_out = n_pool - B + K;
    if (births_out) *births_out = B;
    return GPGMP_OK;
}

}  // namespace gpgmp
