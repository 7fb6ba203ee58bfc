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
//      the cell's first slot in the new pool.  The last tile writes the totals.
//   2. k_pop_move, three independent parts, each writing its own outputs:
//      - every individual of a cell that loses nobody moves to
//        new_start[c] + births[c] + (its rank in the cell);
//      - every cell that loses individuals chooses them uniformly without
//        replacement (Knuth's selection sampling, one Philox draw per candidate while
//        removals remain), writes its survivors in order from new_start[c] and its
//        removed ids to the new pool from kill_off[c]; every cell that gains takes its
//        new ids from the old pool at birth_off[c] and puts them first in the cell;
//      - the unused rest of the old pool follows the removed ids in the new pool.
//   The move kernel first checks the totals against the output capacities and the
//   look-back error word, and writes nothing when a check fails.  The host reads the
//   totals and the check words back once, after both kernels.
// Because the new list is laid out by a scan over the cells, no segmented scan is
// needed: a cell that was empty and a cell that was occupied are placed the same way.
#include <cstdio>
#include <cstring>
#include "common.cuh"
#include "host_common.h"
#include "lookback.cuh"
#include "../../include/gpgmp_c.h"

namespace gpgmp {
namespace {

constexpr int kPlanThreads = 256;
constexpr int kPlanItems = 8;
constexpr int kPlanTile = kPlanThreads * kPlanItems;   // 2048 cells
constexpr int kMoveThreads = 256;

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

__global__ void __launch_bounds__(kPlanThreads)
    k_pop_plan(const uint32_t* __restrict__ count, const int32_t* __restrict__ goal, int64_t ncells,
               uint32_t* __restrict__ new_start, uint32_t* __restrict__ birth_off, uint32_t* __restrict__ kill_off,
               PopHeader* __restrict__ head, uint64_t* __restrict__ status, int64_t tiles) {
    __shared__ uint32_t s_tile;
    __shared__ uint32_t s_warp[3][kPlanThreads / 32];
    __shared__ uint32_t s_prefix[3];
    if (threadIdx.x == 0) s_tile = atomicAdd(&head->tile_counter, 1u);
    __syncthreads();
    const uint32_t tile = s_tile;
    const int64_t base = (int64_t)tile * kPlanTile + (int64_t)threadIdx.x * kPlanItems;
    uint32_t g[kPlanItems], b[kPlanItems], k[kPlanItems];
    uint32_t sum[3] = {0u, 0u, 0u};
    unsigned long long gsum = 0;
#pragma unroll
    for (int q = 0; q < kPlanItems; ++q) {
        uint32_t is = 0, gq = 0;
        if (base + q < ncells) {
            is = __ldg(count + base + q);
            const int32_t g0 = __ldg(goal + base + q);
            gq = g0 > 0 ? (uint32_t)g0 : 0u;
        }
        g[q] = gq;
        b[q] = gq > is ? gq - is : 0u;
        k[q] = is > gq ? is - gq : 0u;
        sum[0] += g[q];
        sum[1] += b[q];
        sum[2] += k[q];
        gsum += gq;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t incl[3] = {sum[0], sum[1], sum[2]};
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
#pragma unroll
        for (int ch = 0; ch < 3; ++ch) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, incl[ch], o);
            if (lane >= o) incl[ch] += t;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) gsum += __shfl_xor_sync(0xffffffffu, gsum, o);
    if (lane == 0 && gsum) atomicAdd(&head->goal_total, gsum);
    if (lane == 31) {
        s_warp[0][warp] = incl[0];
        s_warp[1][warp] = incl[1];
        s_warp[2][warp] = incl[2];
    }
    __syncthreads();
    if (warp < 3) {   // warp ch scans the warp totals of channel ch, then looks back for it
        const int ch = warp;
        uint32_t w = lane < kPlanThreads / 32 ? s_warp[ch][lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += t;
        }
        const uint32_t aggregate = __shfl_sync(0xffffffffu, w, kPlanThreads / 32 - 1);
        if (lane < kPlanThreads / 32) s_warp[ch][lane] = w;   // inclusive over warps
        const uint32_t exclusive =
            warp_lookback_u32(status + (size_t)ch * tiles, tile, aggregate, &head->lookback_err);
        if (lane == 0) {
            s_prefix[ch] = exclusive;
            if ((int64_t)tile == tiles - 1) head->totals[ch] = exclusive + aggregate;
        }
    }
    __syncthreads();
    uint32_t run[3];
#pragma unroll
    for (int ch = 0; ch < 3; ++ch) run[ch] = s_prefix[ch] + (warp ? s_warp[ch][warp - 1] : 0u) + incl[ch] - sum[ch];
#pragma unroll
    for (int q = 0; q < kPlanItems; ++q) {
        if (base + q < ncells) {
            new_start[base + q] = run[0];
            birth_off[base + q] = run[1];
            kill_off[base + q] = run[2];
        }
        run[0] += g[q];
        run[1] += b[q];
        run[2] += k[q];
    }
}

__global__ void __launch_bounds__(kMoveThreads)
    k_pop_move(const uint32_t* __restrict__ keys, const uint32_t* __restrict__ ids, int64_t n,
               const uint32_t* __restrict__ start, const uint32_t* __restrict__ count,
               const int32_t* __restrict__ goal, int64_t ncells, const uint32_t* __restrict__ pool, int64_t n_pool,
               uint32_t seed, uint32_t step, const uint32_t* __restrict__ new_start,
               const uint32_t* __restrict__ birth_off, const uint32_t* __restrict__ kill_off,
               uint32_t* __restrict__ keys_out, uint32_t* __restrict__ ids_out, int64_t capacity_out,
               uint32_t* __restrict__ pool_out, int64_t pool_capacity, PopHeader* __restrict__ head) {
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
    // individuals of cells that lose nobody
    for (int64_t i = t0; i < n; i += stride) {
        const uint32_t c = keys[i];
        if ((int64_t)c >= ncells) continue;
        const uint32_t is = __ldg(count + c);
        const int32_t g0 = __ldg(goal + c);
        const uint32_t g = g0 > 0 ? (uint32_t)g0 : 0u;
        if (is > g) continue;
        const uint32_t o = __ldg(new_start + c) + (g - is) + (uint32_t)(i - __ldg(start + c));
        keys_out[o] = c;
        ids_out[o] = ids[i];
    }
    // cells that lose individuals, and cells that gain
    for (int64_t c = t0; c < ncells; c += stride) {
        const uint32_t is = count[c];
        const int32_t g0 = goal[c];
        const uint32_t g = g0 > 0 ? (uint32_t)g0 : 0u;
        if (is > g) {
            Stream st;
            st.init(seed, 0u, step, (uint32_t)c, PH_POP);
            uint32_t krem = is - g;
            const uint32_t s0 = start[c];
            uint32_t o = new_start[c];
            uint32_t ko = kill_off[c];
            uint32_t i = 0;
            for (; i < is && krem > 0; ++i) {
                // candidate i is removed with probability krem / (is - i)
                const double u = (double)st.next() * (1.0 / 4294967296.0);
                const uint32_t id = ids[s0 + i];
                if ((double)(is - i) * u < (double)krem) {
                    pool_out[ko++] = id;
                    --krem;
                } else {
                    keys_out[o] = (uint32_t)c;
                    ids_out[o++] = id;
                }
            }
            for (; i < is; ++i) {
                keys_out[o] = (uint32_t)c;
                ids_out[o++] = ids[s0 + i];
            }
        } else if (g > is) {
            const uint32_t o = new_start[c], p = birth_off[c];
            for (uint32_t j = 0; j < g - is; ++j) {
                keys_out[o + j] = (uint32_t)c;
                ids_out[o + j] = pool[p + j];
            }
        }
    }
    // the unused rest of the old pool, after the removed ids
    for (int64_t t = t0; t < n_pool - B; t += stride) pool_out[K + t] = pool[B + t];
}

struct PopLayout {
    int64_t tiles;
    size_t head, status, new_start, birth_off, kill_off, bytes;
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
    L.kill_off = o; o = align256(o + 4 * nc);
    L.bytes = o;
    return L;
}

unsigned move_grid(int64_t work) {
    int64_t b = (work + kMoveThreads - 1) / kMoveThreads;
    if (b < 1) b = 1;
    if (b > 148 * 8) b = 148 * 8;
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
    uint32_t* kill_off = (uint32_t*)(base + L.kill_off);
    CK(cudaMemsetAsync(base, 0, L.status + 3 * sizeof(uint64_t) * (size_t)L.tiles, st));
    k_pop_plan<<<(unsigned)L.tiles, kPlanThreads, 0, st>>>(cell_count, goal, ncells, new_start, birth_off, kill_off,
                                                            head, status, L.tiles);
    CK(cudaGetLastError());
    int64_t work = n_active > ncells ? n_active : ncells;
    if (n_pool > work) work = n_pool;
    k_pop_move<<<move_grid(work), kMoveThreads, 0, st>>>(keys, ids, n_active, cell_start, cell_count, goal, ncells,
                                                         pool, n_pool, seed, step, new_start, birth_off, kill_off,
                                                         keys_out, ids_out, cap_out, pool_out, cap_pool, head);
    CK(cudaGetLastError());
    PopHeader h;
    CK(cudaMemcpyAsync(&h, head, sizeof h, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
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
    return GPGMP_OK;
}

}  // extern "C"
