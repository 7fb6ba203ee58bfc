// Individual species on the device (see individual_device.cuh): the prebuilt kernels
// (no model code) and the list operations the solver performs -- build from counts,
// sweep + sort + counts + fields + time step, bookkeeping after a reaction window.
//
// Reference: IndividualSolver.cpp:24-186 (lists and properties), :416-457
// (diffuseX/Y), :458-671 (maintainPopulation), :1083-1153 (sortSpecies,
// computeCellIndices, computeDiffusionConstants); InhomogeneousSolver.cpp:254-427
// (the sweep, then new fields and a new time step for an individual species).
#include <cstdio>
#include <cstring>
#include "individual.h"
#include "host_common.h"
#include "kernels.h"
#include "sort_kernels.h"
#include "../../include/gpgmp_c.h"

namespace gpgmp {
namespace {

constexpr int kIndThreads = 256;

__global__ void __launch_bounds__(kIndThreads) k_ind_sweep(IndArgs a) { ind_sweep_body(a, IndDriftStored()); }
__global__ void __launch_bounds__(kIndThreads) k_ind_fields(IndArgs a) { ind_fields_body(a, IndDriftStored()); }
__global__ void __launch_bounds__(kIndThreads) k_ind_counts(IndArgs a) { ind_counts_body(a); }
__global__ void __launch_bounds__(kIndThreads) k_ind_counts_timestep(IndArgs a, float dx, int kind, float stay,
                                                                     uint32_t* inv_min_key) {
    ind_counts_timestep_body(a, dx, kind, stay, inv_min_key);
}

// goal[r * area + cell] = the species' count in the state
__global__ void k_ind_gather(IndArgs a, int32_t* __restrict__ goal) {
    const long long area = (long long)a.W * a.H, total = (long long)a.R * area;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < total;
         k += (long long)gridDim.x * blockDim.x) {
        const long long r = k / area, cell = k - r * area;
        goal[k] = a.planes[a.species][(r * a.S + a.species) * area + cell];
    }
}

// ids below n0 start with zero properties, the others with DiffusivityX/Y = 1
// (IndividualSolver.cpp:52-98)
__global__ void k_ind_props_init(float* __restrict__ props, long long cap, long long n0) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < cap;
         i += (long long)gridDim.x * blockDim.x) {
        const float d = i < n0 ? 0.f : 1.f;
        props[i] = d;
        props[cap + i] = d;
        props[2 * cap + i] = 0.f;
        props[3 * cap + i] = 0.f;
    }
}

__global__ void k_ind_iota(uint32_t* __restrict__ v, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        v[i] = (uint32_t)i;
}

// the first `births` ids of the old pool are the new individuals
__global__ void k_ind_mark(const uint32_t* __restrict__ pool, long long births, uint8_t* __restrict__ newborn) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < births;
         i += (long long)gridDim.x * blockDim.x)
        newborn[pool[i]] = 1;
}

unsigned grid_for(long long work) {
    long long b = (work + kIndThreads - 1) / kIndThreads;
    if (b < 1) b = 1;
    if (b > 148 * 8) b = 148 * 8;
    return (unsigned)b;
}

int bits_for(uint32_t max_key) {
    int b = 1;
    while (b < 32 && (max_key >> b) != 0) ++b;
    return b;
}

#define CK(expr)                                                                                           \
    do {                                                                                                   \
        cudaError_t e_ = (expr);                                                                           \
        if (e_ != cudaSuccess) return set_error(GPGMP_ERR_CUDA, "%s: %s", #expr, cudaGetErrorString(e_)); \
    } while (0)

cudaError_t run_sweep(const IndKernels& k, const IndArgs& a, cudaStream_t st) {
    if (a.n <= 0) return cudaSuccess;
    if (k.sweep) return launch_ind_jit(k.sweep, a, a.n, st);
    k_ind_sweep<<<grid_for(a.n), kIndThreads, 0, st>>>(a);
    return cudaGetLastError();
}

cudaError_t run_fields(const IndKernels& k, const IndArgs& a, cudaStream_t st) {
    const long long total = (long long)a.R * a.W * a.H;
    if (k.fields) return launch_ind_jit(k.fields, a, total, st);
    k_ind_fields<<<grid_for(total), kIndThreads, 0, st>>>(a);
    return cudaGetLastError();
}

void bind(IndList& l, IndArgs& a) {
    a.keys = l.keys[l.cur];
    a.ids = l.ids[l.cur];
    a.n = l.n;
    a.killed_key = (uint32_t)l.ncells;
    a.props = l.props;
    a.cap = l.cap;
    a.start = l.start[0];
    a.count = l.count;
    a.fDx = l.fields;
    a.fDy = l.fields + l.ncells;
    a.fRx = l.fields + 2 * l.ncells;
    a.fRy = l.fields + 3 * l.ncells;
    a.newborn = l.newborn;
    a.killed = l.d_small;
}

}  // namespace

int ind_alloc(IndList& l, int species, long long cap, long long ncells, bool may_leave) {
    ind_free(l);
    l.species = species;
    l.cap = cap > 0 ? cap : 1;
    l.ncells = ncells;
    // the killed key (ncells) only occurs with an absorbing wall: without one the sort
    // needs the bits of the last cell only
    l.key_bits = bits_for((uint32_t)(may_leave ? ncells : ncells - 1));
    l.sort_bytes = sort_layout(l.cap, l.key_bits).bytes;
    l.scan_bytes = scan_scratch_bytes(ncells + 1);
    l.pop_bytes = 0;
    if (gpgmp_population_scratch_bytes(l.cap, ncells + 1, &l.pop_bytes) != GPGMP_OK) return GPGMP_ERR_INVALID;
    const size_t b = sizeof(uint32_t) * (size_t)l.cap;
    const size_t cb = sizeof(uint32_t) * (size_t)(ncells + 1);
    cudaError_t e = cudaSuccess;
    auto A = [&](void** p, size_t bytes) {
        if (e == cudaSuccess) e = cudaMalloc(p, bytes > 0 ? bytes : 1);
    };
    for (int i = 0; i < 2; ++i) {
        A((void**)&l.keys[i], b);
        A((void**)&l.ids[i], b);
        A((void**)&l.pool[i], b);
        A((void**)&l.start[i], cb);
    }
    A((void**)&l.props, 4 * sizeof(float) * (size_t)l.cap);
    A((void**)&l.newborn, (size_t)l.cap);
    A((void**)&l.goal, cb);
    // count, fields and the two result words in one block, so that a sweep clears them
    // with one memset
    const size_t cb_al = (cb + 255) & ~(size_t)255;
    const size_t fb_al = (4 * sizeof(float) * (size_t)ncells + 255) & ~(size_t)255;
    A(&l.sweep_block, cb_al + fb_al + 2 * sizeof(uint32_t));
    if (e == cudaSuccess) {
        l.count = (uint32_t*)l.sweep_block;
        l.fields = (float*)((char*)l.sweep_block + cb_al);
        l.d_small = (uint32_t*)((char*)l.sweep_block + cb_al + fb_al);
        e = cudaMallocHost((void**)&l.h_small, 4 * sizeof(uint32_t));
    }
    A(&l.sort_scratch, l.sort_bytes);
    A(&l.scan_scratch, l.scan_bytes);
    A(&l.pop_scratch, l.pop_bytes);
    if (e == cudaSuccess) e = cudaMemset(l.newborn, 0, (size_t)l.cap);
    if (e == cudaSuccess) e = cudaMemset(l.count, 0, cb);
    if (e == cudaSuccess) e = cudaMemset(l.start[0], 0, cb);
    if (e != cudaSuccess) {
        ind_free(l);
        return set_error(e == cudaErrorMemoryAllocation ? GPGMP_ERR_NOMEM : GPGMP_ERR_CUDA, "individual lists: %s",
                         cudaGetErrorString(e));
    }
    return GPGMP_OK;
}

void ind_free(IndList& l) {
    void* ptrs[] = {l.keys[0], l.keys[1], l.ids[0],  l.ids[1],       l.pool[0],      l.pool[1],
                    l.start[0], l.start[1], l.props, l.newborn, l.goal,         l.sweep_block,
                    l.sort_scratch, l.scan_scratch, l.pop_scratch};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (l.h_small) cudaFreeHost(l.h_small);
    const int sp = l.species;
    l = IndList();
    l.species = sp;
}

int ind_sort(IndList& l, cudaStream_t st) {
    if (l.sorted) return GPGMP_OK;
    const int c = l.cur;
    // the sort's last pass counts the individuals per key (cells and the killed bin)
    CK(cudaMemsetAsync(l.count, 0, sizeof(uint32_t) * (size_t)(l.ncells + 1), st));
    if (l.n > 0) {
        CK(radix_sort_pairs_u32(l.keys[c], l.ids[c], l.keys[1 - c], l.ids[1 - c], l.n, l.key_bits, l.sort_scratch, st,
                                l.count, l.ncells + 1));
        l.cur = 1 - c;
    }
    CK(scan_exclusive_u32(l.count, l.start[0], l.ncells + 1, l.scan_scratch, st));
    uint32_t err[2] = {0, 0};
    CK(cudaMemcpyAsync(&err[0], (const char*)l.scan_scratch + scan_error_flag_offset(), sizeof(uint32_t),
                       cudaMemcpyDeviceToHost, st));
    if (l.n > 0)
        CK(cudaMemcpyAsync(&err[1], (const char*)l.sort_scratch + sort_layout(l.n, l.key_bits).off_counters + 16,
                           sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    if (l.pending > 0) {
        // the ones that left sort last: their ids go to the end of the pool
        const long long alive = l.n - l.pending;
        CK(cudaMemcpyAsync(l.pool[l.pcur] + l.npool, l.ids[l.cur] + alive, sizeof(uint32_t) * (size_t)l.pending,
                           cudaMemcpyDeviceToDevice, st));
        l.npool += l.pending;
        l.n = alive;
        l.pending = 0;
        CK(cudaMemsetAsync(l.count + l.ncells, 0, sizeof(uint32_t), st));
    }
    CK(cudaStreamSynchronize(st));
    if (err[0] || err[1]) return set_error(GPGMP_ERR_TIMEOUT, "a look-back wait of the sort or scan gave up");
    l.sorted = true;
    return GPGMP_OK;
}

int ind_fields(IndList& l, IndArgs a, const IndKernels& k, cudaStream_t st) {
    int rc = ind_sort(l, st);
    if (rc) return rc;
    bind(l, a);
    CK(run_fields(k, a, st));
    return GPGMP_OK;
}

int ind_build(IndList& l, IndArgs a, const IndKernels& k, cudaStream_t st) {
    bind(l, a);
    k_ind_gather<<<grid_for(l.ncells), kIndThreads, 0, st>>>(a, l.goal);
    CK(cudaGetLastError());
    CK(cudaMemsetAsync(l.goal + l.ncells, 0, sizeof(int32_t), st));
    l.pcur = 0;
    k_ind_iota<<<grid_for(l.cap), kIndThreads, 0, st>>>(l.pool[0], l.cap);
    CK(cudaGetLastError());
    CK(cudaMemsetAsync(l.count, 0, sizeof(uint32_t) * (size_t)(l.ncells + 1), st));
    CK(cudaMemsetAsync(l.start[0], 0, sizeof(uint32_t) * (size_t)(l.ncells + 1), st));
    l.n = 0;
    l.npool = l.cap;
    int64_t n_new = 0, np_new = 0;
    const int c = l.cur;
    int rc = population_maintain(nullptr, nullptr, 0, l.start[0], l.count, l.goal, l.ncells + 1, l.pool[0], l.npool,
                                 a.seed, a.step_seed, l.keys[1 - c], l.ids[1 - c], l.cap, l.pool[1], l.cap,
                                 l.start[1], &n_new, &np_new, nullptr, l.pop_scratch, l.pop_bytes, st);
    if (rc == GPGMP_ERR_INVALID)
        return set_error(GPGMP_ERR_INVALID, "species %d: more individuals than the capacity %lld", l.species,
                         (long long)l.cap);
    if (rc) return rc;
    l.cur = 1 - c;
    l.pcur = 1;
    l.n = n_new;
    l.npool = np_new;
    std::swap(l.start[0], l.start[1]);
    CK(cudaMemcpyAsync(l.count, l.goal, sizeof(uint32_t) * (size_t)(l.ncells + 1), cudaMemcpyDeviceToDevice, st));
    k_ind_props_init<<<grid_for(l.cap), kIndThreads, 0, st>>>(l.props, l.cap, l.n);
    CK(cudaGetLastError());
    return ind_fields(l, a, k, st);
}

int ind_sweep(IndList& l, IndArgs a, const IndKernels& k, float dx, int ts_kind, float stay, int slot,
              cudaStream_t st) {
    bind(l, a);
    // count, fields, the departures word and the inverted time step key
    CK(cudaMemsetAsync(l.sweep_block, 0, (size_t)((char*)(l.d_small + 2) - (char*)l.sweep_block), st));
    CK(run_sweep(k, a, st));
    l.sorted = false;
    k_ind_counts_timestep<<<grid_for(l.ncells), kIndThreads, 0, st>>>(a, dx, ts_kind, stay, l.d_small + 1);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(l.h_small + 2 * slot, l.d_small, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    return GPGMP_OK;
}

float ind_sweep_result(IndList& l, int slot) {
    l.pending += l.h_small[2 * slot];
    return key_to_float(~l.h_small[2 * slot + 1]);
}

int ind_maintain(IndList& l, IndArgs a, const IndKernels& k, cudaStream_t st) {
    int rc0 = ind_sort(l, st);
    if (rc0) return rc0;
    bind(l, a);
    k_ind_gather<<<grid_for(l.ncells), kIndThreads, 0, st>>>(a, l.goal);
    CK(cudaGetLastError());
    CK(cudaMemsetAsync(l.goal + l.ncells, 0, sizeof(int32_t), st));
    int64_t n_new = 0, np_new = 0, births = 0;
    const int c = l.cur, p = l.pcur;
    int rc = population_maintain(l.n ? l.keys[c] : nullptr, l.n ? l.ids[c] : nullptr, l.n, l.start[0], l.count,
                                 l.goal, l.ncells + 1, l.npool ? l.pool[p] : nullptr, l.npool, a.seed, a.step_seed,
                                 l.keys[1 - c], l.ids[1 - c], l.cap, l.pool[1 - p], l.cap, l.start[1], &n_new, &np_new,
                                 &births, l.pop_scratch, l.pop_bytes, st);
    if (rc == GPGMP_ERR_INVALID)
        return set_error(GPGMP_ERR_INVALID, "species %d: more individuals than the capacity %lld", l.species,
                         (long long)l.cap);
    if (rc) return rc;
    if (k.newborn_active && births > 0) {
        k_ind_mark<<<grid_for(births), kIndThreads, 0, st>>>(l.pool[p], births, l.newborn);
        CK(cudaGetLastError());
    }
    l.cur = 1 - c;
    l.pcur = 1 - p;
    l.n = n_new;
    l.npool = np_new;
    std::swap(l.start[0], l.start[1]);
    CK(cudaMemcpyAsync(l.count, l.goal, sizeof(uint32_t) * (size_t)(l.ncells + 1), cudaMemcpyDeviceToDevice, st));
    if (k.newborn_active && births > 0) {
        bind(l, a);
        CK(launch_ind_jit(k.newborn, a, l.n, st));
    }
    return GPGMP_OK;
}

}  // namespace gpgmp
