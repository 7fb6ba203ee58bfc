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
//   bin:     stable radix sort of (key, index), count per cell, exclusive scan;
//   react:   in each cell the k-th A (in sorted order) pairs with the k-th B and the
//            pair is removed with probability p (one 32-bit draw per pair against
//            floor(p 2^32));
//   compact: survivors in sorted order (exclusive scan of the alive flags).
// Compiled with -fmad=false: positions must round as the CPU replay does.
#include <cmath>
#include <cstdint>
#include <cuda_runtime.h>
#include "common.cuh"
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

__global__ void k_move(float* __restrict__ px, float* __restrict__ py, int64_t n, int G, float sig, float ax, float ay,
                       uint32_t seed, uint32_t step, uint32_t* __restrict__ keys, uint32_t* __restrict__ vals) {
    const float L = (float)G;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
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
        keys[i] = (uint32_t)(int)y * (uint32_t)G + (uint32_t)(int)x;
        vals[i] = (uint32_t)i;
    }
}

__global__ void k_fill_u32(uint32_t* p, int64_t n, uint32_t v) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        p[i] = v;
}

__global__ void k_react(const uint32_t* __restrict__ start, const uint32_t* __restrict__ count, int64_t ncells,
                        const uint32_t* __restrict__ svals, const uint8_t* __restrict__ sp, uint32_t seed,
                        uint32_t step, uint32_t thresh, uint32_t* __restrict__ alive) {
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < ncells;
         c += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t cnt = count[c];
        if (cnt < 2) continue;
        const uint32_t s0 = start[c], e = s0 + cnt;
        Stream st;
        st.init(seed, 1u, step, (uint32_t)c, PH_PAIR);
        uint32_t ia = s0, ib = s0;
        for (;;) {
            while (ia < e && sp[svals[ia]] != 0) ia++;
            while (ib < e && sp[svals[ib]] != 1) ib++;
            if (ia >= e || ib >= e) break;
            const uint32_t u = st.next();
            if (u < thresh) {
                alive[ia] = 0;
                alive[ib] = 0;
            }
            ia++;
            ib++;
        }
    }
}

__global__ void k_gather(const uint32_t* __restrict__ alive, const uint32_t* __restrict__ pos,
                         const uint32_t* __restrict__ svals, int64_t n, const float* __restrict__ x,
                         const float* __restrict__ y, const uint8_t* __restrict__ sp, float* __restrict__ x2,
                         float* __restrict__ y2, uint8_t* __restrict__ sp2) {
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x) {
        if (!alive[j]) continue;
        const uint32_t d = pos[j], s = svals[j];
        x2[d] = x[s];
        y2[d] = y[s];
        sp2[d] = sp[s];
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
    uint32_t *start = nullptr, *count = nullptr, *alive = nullptr, *pos = nullptr;
    void *sort_scratch = nullptr, *scan_scratch = nullptr;
    uint32_t* host_tail = nullptr;   // pinned: last scan value and last flag
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
                    h->count, h->alive, h->pos, h->sort_scratch, h->scan_scratch};
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
    A((void**)&h->alive, n4); A((void**)&h->pos, n4);
    A((void**)&h->start, sizeof(uint32_t) * (size_t)ncells); A((void**)&h->count, sizeof(uint32_t) * (size_t)ncells);
    A(&h->sort_scratch, sort_layout(capacity, bits).bytes);
    const int64_t scan_n = capacity > ncells ? capacity : ncells;
    A(&h->scan_scratch, scan_scratch_bytes(scan_n));
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
    if (n > 0) {
        k_move<<<grid_of(n, 256), 256, 0, st>>>(h->x, h->y, n, h->grid, sig, ax, ay, h->seed, step, h->keys, h->vals);
        CK(cudaGetLastError());
        CK(radix_sort_pairs_u32(h->keys, h->vals, h->skeys, h->svals, n, h->key_bits, h->sort_scratch, st));
    }
    CK(cell_offsets_u32(h->skeys, n, ncells, h->start, h->count, h->scan_scratch, st));
    if (n > 0) {
        k_fill_u32<<<grid_of(n, 256), 256, 0, st>>>(h->alive, n, 1u);
        k_react<<<grid_of(ncells, 128), 128, 0, st>>>(h->start, h->count, ncells, h->svals, h->sp, h->seed, step,
                                                       h->thresh, h->alive);
        CK(cudaGetLastError());
        CK(scan_exclusive_u32(h->alive, h->pos, n, h->scan_scratch, st));
        k_gather<<<grid_of(n, 256), 256, 0, st>>>(h->alive, h->pos, h->svals, n, h->x, h->y, h->sp, h->x2, h->y2,
                                                   h->sp2);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(&h->host_tail[0], h->pos + n - 1, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(&h->host_tail[1], h->alive + n - 1, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        h->n = (int64_t)h->host_tail[0] + h->host_tail[1];
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
    CK(cudaMemcpy(&b, (const char*)h->scan_scratch + scan_error_flag_offset(), sizeof(int), cudaMemcpyDeviceToHost));
    *status = (a || b) ? GPGMP_ERR_TIMEOUT : GPGMP_OK;
    return GPGMP_OK;
}

}  // extern "C"
