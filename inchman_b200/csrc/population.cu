// Individual-particle population bookkeeping: after a reaction window changed the
// per-cell counts, bring the cell-sorted list of individuals back in line with them.
//
// The reference does this with maintainPopulation, a segmented scan over the grid,
// reduction offsets over the particle list, scatter / new-particle / lost-particle
// kernels and a final copy (IndividualSolver.cpp:458-671, IndividualSolver.cl:
// 1017-1882, doc/source/individual.rst).  Here the same result comes from three
// exclusive scans (decoupled look-back, sort.cu) and three gather/scatter kernels:
//   1. per cell: is = current count, goal = target count; kills = is - goal chosen
//      uniformly without replacement among the cell's individuals (Knuth's selection
//      sampling, one Philox draw per candidate), births = goal - is;
//   2. scans: of goal (the new cell starts), of births (pool positions), of the kill
//      flags over the list (pool positions of the killed ids);
//   3. survivors move to new_start[c] + births[c] + (their rank among the cell's
//      survivors); the cell's births come first, with ids taken from the front of the
//      pool in cell order; the new pool is the killed ids (in list order) followed by
//      the unused rest of the old pool.
// Because the new list is laid out by a scan over the cells, no segmented scan is
// needed: a cell that was empty and a cell that was occupied are placed the same way.
#include <cstdio>
#include <cstring>
#include "common.cuh"
#include "host_common.h"
#include "sort_kernels.h"
#include "../../include/gpgmp_c.h"

namespace gpgmp {
namespace {

__global__ void k_pop_decide(const uint32_t* __restrict__ start, const uint32_t* __restrict__ count,
                             const int32_t* __restrict__ goal, int64_t ncells, uint32_t seed, uint32_t step,
                             uint32_t* __restrict__ goal_u, uint32_t* __restrict__ births,
                             uint32_t* __restrict__ dead) {
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < ncells;
         c += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t is = count[c];
        const int32_t g0 = goal[c];
        const uint32_t g = g0 > 0 ? (uint32_t)g0 : 0u;
        goal_u[c] = g;
        births[c] = g > is ? g - is : 0u;
        if (is > g) {
            // selection sampling: candidate i is taken with probability k_rem / (is - i)
            Stream st;
            st.init(seed, 0u, step, (uint32_t)c, PH_POP);
            uint32_t krem = is - g;
            const uint32_t s0 = start[c];
            for (uint32_t i = 0; i < is && krem > 0; ++i) {
                const double u = (double)st.next() * (1.0 / 4294967296.0);
                if ((double)(is - i) * u < (double)krem) {
                    dead[s0 + i] = 1u;
                    --krem;
                }
            }
        }
    }
}

__global__ void k_pop_scatter(const uint32_t* __restrict__ keys, const uint32_t* __restrict__ ids, int64_t n,
                              const uint32_t* __restrict__ start, const uint32_t* __restrict__ dead,
                              const uint32_t* __restrict__ kill_pos, const uint32_t* __restrict__ new_start,
                              const uint32_t* __restrict__ births, uint32_t* __restrict__ keys_out,
                              uint32_t* __restrict__ ids_out, uint32_t* __restrict__ pool_out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        if (dead[i]) {
            pool_out[kill_pos[i]] = ids[i];
            continue;
        }
        const uint32_t c = keys[i];
        const uint32_t s0 = start[c];
        const uint32_t rank = (uint32_t)(i - s0) - (kill_pos[i] - kill_pos[s0]);
        const uint32_t o = new_start[c] + births[c] + rank;
        keys_out[o] = c;
        ids_out[o] = ids[i];
    }
}

__global__ void k_pop_births(const uint32_t* __restrict__ births, const uint32_t* __restrict__ birth_off,
                             const uint32_t* __restrict__ new_start, int64_t ncells, const uint32_t* __restrict__ pool,
                             uint32_t* __restrict__ keys_out, uint32_t* __restrict__ ids_out) {
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < ncells;
         c += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t b = births[c];
        for (uint32_t j = 0; j < b; ++j) {
            keys_out[new_start[c] + j] = (uint32_t)c;
            ids_out[new_start[c] + j] = pool[birth_off[c] + j];
        }
    }
}

__global__ void k_pop_pool_tail(const uint32_t* __restrict__ pool, int64_t from, int64_t count,
                                uint32_t* __restrict__ pool_out, int64_t to) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < count; t += (int64_t)gridDim.x * blockDim.x)
        pool_out[to + t] = pool[from + t];
}

unsigned grid_of(int64_t n) {
    int64_t b = (n + 255) / 256;
    if (b < 1) b = 1;
    if (b > 148 * 16) b = 148 * 16;
    return (unsigned)b;
}

struct PopLayout {
    size_t dead, kill_pos, goal_u, births, birth_off, new_start, scan[3], bytes;
};

size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

PopLayout pop_layout(int64_t n, int64_t ncells) {
    PopLayout L;
    size_t o = 0;
    const size_t nn = (size_t)(n > 0 ? n : 1), nc = (size_t)ncells;
    L.dead = o; o = align256(o + 4 * nn);
    L.kill_pos = o; o = align256(o + 4 * nn);
    L.goal_u = o; o = align256(o + 4 * nc);
    L.births = o; o = align256(o + 4 * nc);
    L.birth_off = o; o = align256(o + 4 * nc);
    L.new_start = o; o = align256(o + 4 * nc);
    // one scan scratch each, so that a look-back error word of one is not cleared by the next
    L.scan[0] = o; o = align256(o + scan_scratch_bytes(ncells));
    L.scan[1] = o; o = align256(o + scan_scratch_bytes(ncells));
    L.scan[2] = o; o = align256(o + scan_scratch_bytes(n > 0 ? n : 1));
    L.bytes = o;
    return L;
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
    *bytes = pop_layout(n_active, ncells).bytes;
    return GPGMP_OK;
}

int gpgmp_population_maintain(const uint32_t* keys, const uint32_t* ids, int64_t n_active, const uint32_t* cell_start,
                              const uint32_t* cell_count, const int32_t* goal, int64_t ncells, const uint32_t* pool,
                              int64_t n_pool, uint32_t seed, uint32_t step, uint32_t* keys_out, uint32_t* ids_out,
                              int64_t capacity_out, uint32_t* pool_out, int64_t pool_capacity, uint32_t* start_out,
                              int64_t* n_active_out, int64_t* n_pool_out, void* scratch, size_t scratch_bytes,
                              void* stream) {
    if (n_active < 0 || n_pool < 0 || ncells <= 0 || n_active >= ((int64_t)1 << 31) || ncells >= ((int64_t)1 << 31))
        return set_error(GPGMP_ERR_INVALID, "bad sizes");
    if (!cell_start || !cell_count || !goal || !keys_out || !ids_out || !pool_out || !n_active_out || !n_pool_out ||
        !scratch || (n_active > 0 && (!keys || !ids)) || (n_pool > 0 && !pool))
        return set_error(GPGMP_ERR_INVALID, "NULL argument");
    const PopLayout L = pop_layout(n_active, ncells);
    if (scratch_bytes < L.bytes) return set_error(GPGMP_ERR_INVALID, "scratch too small");
    cudaStream_t st = (cudaStream_t)stream;
    char* base = (char*)scratch;
    uint32_t* dead = (uint32_t*)(base + L.dead);
    uint32_t* kill_pos = (uint32_t*)(base + L.kill_pos);
    uint32_t* goal_u = (uint32_t*)(base + L.goal_u);
    uint32_t* births = (uint32_t*)(base + L.births);
    uint32_t* birth_off = (uint32_t*)(base + L.birth_off);
    uint32_t* new_start = start_out ? start_out : (uint32_t*)(base + L.new_start);
    void* scan[3] = {base + L.scan[0], base + L.scan[1], base + L.scan[2]};
    if (n_active > 0) CK(cudaMemsetAsync(dead, 0, sizeof(uint32_t) * n_active, st));
    k_pop_decide<<<grid_of(ncells), 256, 0, st>>>(cell_start, cell_count, goal, ncells, seed, step, goal_u, births,
                                                  dead);
    CK(cudaGetLastError());
    CK(scan_exclusive_u32(goal_u, new_start, ncells, scan[0], st));
    CK(scan_exclusive_u32(births, birth_off, ncells, scan[1], st));
    if (n_active > 0) CK(scan_exclusive_u32(dead, kill_pos, n_active, scan[2], st));
    // totals: new active count, births, kills (exclusive scan + last element)
    uint32_t h[6] = {0, 0, 0, 0, 0, 0};
    CK(cudaMemcpyAsync(&h[0], new_start + ncells - 1, 4, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(&h[1], goal_u + ncells - 1, 4, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(&h[2], birth_off + ncells - 1, 4, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(&h[3], births + ncells - 1, 4, cudaMemcpyDeviceToHost, st));
    if (n_active > 0) {
        CK(cudaMemcpyAsync(&h[4], kill_pos + n_active - 1, 4, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(&h[5], dead + n_active - 1, 4, cudaMemcpyDeviceToHost, st));
    }
    CK(cudaStreamSynchronize(st));
    for (int q = 0; q < (n_active > 0 ? 3 : 2); ++q) {     // the third scan ran only for a non-empty list
        int err = 0;
        CK(cudaMemcpy(&err, (const char*)scan[q] + scan_error_flag_offset(), sizeof(int), cudaMemcpyDeviceToHost));
        if (err) return set_error(GPGMP_ERR_TIMEOUT, "a scan's look-back wait gave up");
    }
    const int64_t n_new = (int64_t)h[0] + h[1], B = (int64_t)h[2] + h[3], K = (int64_t)h[4] + h[5];
    if (B > n_pool)
        return set_error(GPGMP_ERR_INVALID, "%lld new individuals but only %lld free ids", (long long)B,
                         (long long)n_pool);
    if (n_new > capacity_out) return set_error(GPGMP_ERR_INVALID, "output list holds %lld of %lld individuals",
                                               (long long)capacity_out, (long long)n_new);
    const int64_t p_new = n_pool - B + K;
    if (p_new > pool_capacity) return set_error(GPGMP_ERR_INVALID, "output pool too small");
    if (n_active > 0) {
        k_pop_scatter<<<grid_of(n_active), 256, 0, st>>>(keys, ids, n_active, cell_start, dead, kill_pos, new_start,
                                                         births, keys_out, ids_out, pool_out);
        CK(cudaGetLastError());
    }
    k_pop_births<<<grid_of(ncells), 256, 0, st>>>(births, birth_off, new_start, ncells, pool, keys_out, ids_out);
    CK(cudaGetLastError());
    if (n_pool - B > 0) {
        k_pop_pool_tail<<<grid_of(n_pool - B), 256, 0, st>>>(pool, B, n_pool - B, pool_out, K);
        CK(cudaGetLastError());
    }
    *n_active_out = n_new;
    *n_pool_out = p_new;
    return GPGMP_OK;
}

}  // extern "C"
