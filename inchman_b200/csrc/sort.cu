// Scan, radix sort and cell offsets of the individual-particle path.
//
// Reference: IndividualSolver sorts (cell, id) pairs with an LSD radix sort of
// 4-bit digits built from block sort / radix offsets / 3-kernel exclusive scan /
// reorder, 6 synchronous launches per pass and 8 passes (IndividualSolver.cpp:673-808,
// kernels IndividualSolver.cl:36-369, 493-553), then derives each cell's first and
// last particle (computeCellIndices, IndividualSolver.cl:564-619).  The result is
// the stable sort by cell.
//
// Here, from the published methods (not from the reference's SDK-derived code):
//  - exclusive scan: single pass with decoupled look-back (Merrill & Garland 2016);
//  - radix sort: onesweep (Adinets & Merrill 2022): one histogram kernel for every
//    digit position, then one kernel per digit (8 bits, or 10 where that saves a
//    pass: 17-20 and 25-30 key bits) that ranks its tile (peer masks from shared-memory
//    atomicOr on the digit's low 8 bits, ballots for the rest),
//    publishes per-digit tile counts, looks back for the prefix and scatters through
//    shared memory; tile 0 scans the pass's digit counts into the digits' global
//    starts and publishes them inside its inclusive prefix, so no other tile (and no
//    separate launch) turns counts into offsets; stable;
//  - cell offsets: key histogram + exclusive scan (start), count; the reference's
//    left/right indices follow from them.
// Every look-back spin has an iteration limit; exceeding it sets the error word
// (GPGMP_ERR_TIMEOUT for the caller) and the kernel continues without waiting.
#include <algorithm>
#include <cstdint>
#include <mutex>
#include <cuda_runtime.h>
#include "lookback.cuh"
#include "sort_kernels.h"
#include "host_common.h"
#include "../../include/gpgmp_c.h"

namespace gpgmp {
namespace {

constexpr int kScanThreads = 512;
constexpr int kScanItems = 32;
constexpr int kScanTile = kScanThreads * kScanItems;   // 16384

// ---- exclusive scan ------------------------------------------------------------
// scratch: [0] tile counter, [1] error word, then one status word per tile:
// (flag << 32) | value, flag 0 = not ready, 1 = tile aggregate, 2 = inclusive prefix.
// A tile is 512 threads x 32 consecutive values (16384: fewer tiles, a shorter
// look-back chain).  Every tile moves through shared memory, one uint4 of padding per
// eight so that a thread's 128-byte row reads and writes without bank conflicts: a
// full tile whose pointers are 16-byte aligned (vec) with warp-contiguous 16-byte loads
// and stores (every HBM request coalesced), a partial tile or unaligned pointers with
// coalesced element loads and stores.  A thread sums its row from shared memory, and
// after the look-back writes its row's exclusive prefixes back in place: the values
// never sit in registers, so three CTAs fit on an SM (shared memory is the limit)
// instead of two (registers were), and more loads are in flight while tiles wait in
// the look-back.
constexpr int kScanQuads = kScanTile / 4;                 // uint4 per tile
__device__ __forceinline__ int scan_pad(int i4) { return i4 + (i4 >> 3); }
// word index of value i of the tile in the padded layout
__device__ __forceinline__ int scan_word(int i) { return 4 * scan_pad(i >> 2) + (i & 3); }

__global__ void __launch_bounds__(kScanThreads, 3) k_scan_exclusive(const uint32_t* __restrict__ in,
                                                                    uint32_t* __restrict__ out, int64_t n,
                                                                    uint64_t* __restrict__ scratch, int vec) {
    extern __shared__ uint4 s_io[];   // kScanQuads + kScanQuads / 8 (dynamic: 72 KB)
    uint32_t* s_w32 = reinterpret_cast<uint32_t*>(s_io);
    __shared__ uint32_t s_tile;
    __shared__ uint32_t s_warp[kScanThreads / 32];
    __shared__ uint32_t s_prefix;
    unsigned int* counter = reinterpret_cast<unsigned int*>(scratch);
    int* err = reinterpret_cast<int*>(scratch) + 2;
    uint64_t* status = scratch + 2;
    if (threadIdx.x == 0) s_tile = atomicAdd(counter, 1u);
    __syncthreads();
    const uint32_t tile = s_tile;
    const int64_t tbase = (int64_t)tile * kScanTile;
    const bool full = vec && tbase + kScanTile <= n;    // the same in every thread of the block
    if (full) {
        const uint4* src = reinterpret_cast<const uint4*>(in + tbase);
#pragma unroll
        for (int q = 0; q < kScanItems / 4; ++q) {
            const int i4 = q * kScanThreads + threadIdx.x;
            s_io[scan_pad(i4)] = src[i4];
        }
    } else {
        for (int q = 0; q < kScanItems; ++q) {
            const int i = q * kScanThreads + threadIdx.x;
            s_w32[scan_word(i)] = tbase + i < n ? in[tbase + i] : 0u;
        }
    }
    __syncthreads();
    // the thread's row: values threadIdx.x * 32 .. + 31 of the tile
    const int row = threadIdx.x * (kScanItems / 4);
    uint32_t sum = 0;
#pragma unroll
    for (int q = 0; q < kScanItems / 4; ++q) {
        const uint4 w = s_io[scan_pad(row + q)];
        sum += w.x + w.y + w.z + w.w;
    }
    // block exclusive scan of the thread sums
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < kScanThreads / 32 ? s_warp[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t t = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += t;
        }
        if (lane < kScanThreads / 32) s_warp[lane] = w;   // inclusive over warps
    }
    __syncthreads();
    const uint32_t warp_excl = warp == 0 ? 0u : s_warp[warp - 1];
    const uint32_t thread_excl = warp_excl + incl - sum;
    const uint32_t aggregate = s_warp[kScanThreads / 32 - 1];
    // decoupled look-back by warp 0
    if (warp == 0) {
        const uint32_t exclusive = warp_lookback_u32(status, tile, aggregate, err);
        if (lane == 0) s_prefix = exclusive;
    }
    __syncthreads();
    // the row's exclusive prefixes, in place
    uint32_t run = s_prefix + thread_excl;
#pragma unroll
    for (int q = 0; q < kScanItems / 4; ++q) {
        const uint4 v = s_io[scan_pad(row + q)];
        uint4 w;
        w.x = run; run += v.x;
        w.y = run; run += v.y;
        w.z = run; run += v.z;
        w.w = run; run += v.w;
        s_io[scan_pad(row + q)] = w;
    }
    __syncthreads();
    if (full) {
        uint4* dst = reinterpret_cast<uint4*>(out + tbase);
#pragma unroll
        for (int q = 0; q < kScanItems / 4; ++q) {
            const int i4 = q * kScanThreads + threadIdx.x;
            dst[i4] = s_io[scan_pad(i4)];
        }
    } else {
        for (int q = 0; q < kScanItems; ++q) {
            const int i = q * kScanThreads + threadIdx.x;
            if (tbase + i < n) out[tbase + i] = s_w32[scan_word(i)];
        }
    }
}

// ---- radix sort ------------------------------------------------------------------
// A tile is kThreads threads x kSortItems keys.  8-bit passes run 256-thread tiles, four
// CTAs per SM (one CTA's barriers overlap the others' work); 10-bit passes 512-thread
// tiles, two per SM (with 256 threads each would own four digits and spill registers).
constexpr int kSortItems = 15;
template <int RB>
struct SortShape {
    static constexpr int kThreads = RB == 8 ? 256 : 512;
    static constexpr int kMinBlocks = RB == 8 ? 4 : 2;
    static constexpr int kTile = kThreads * kSortItems;   // 3840 / 7680 keys
    static constexpr int kWarps = kThreads / 32;
    // keys and values of a tile in sorted order (dynamic shared memory: 30 / 60 KB)
    static constexpr int kStagingBytes = 2 * kTile * (int)sizeof(uint32_t);
    static_assert(kThreads >= 256 && kThreads % 32 == 0, "a thread per digit (8-bit digits)");
};
// 8-bit passes copy the values asynchronously into the values' staging area while the
// tile ranks and stage them in two steps (through registers); 10-bit passes read them at
// the staging step, which measured faster for them than the extra barrier of the
// two-step form.
template <int RB>
constexpr bool kValuePrefetch = RB == 8;
constexpr uint32_t kFlagA = 1u << 30, kFlagP = 2u << 30, kValMask = (1u << 30) - 1;
constexpr int kLookWindow = 4;   // predecessor tiles read per look-back step
constexpr int kHistWords = 3 * 1024;   // digit counts of every pass: 4 x 256 or up to 3 x 1024

// Digits of RB bits: DIG values, owned kDPT at a time by the first kDigitThreads threads
// in the digit phases (8 bits: all 256 threads, one each; 10 bits: all 512, two each).
template <int RB>
struct Radix {
    static constexpr int DIG = 1 << RB;
    static constexpr uint32_t MASK = (uint32_t)DIG - 1u;
    static constexpr int kDigitThreads = DIG < SortShape<RB>::kThreads ? DIG : SortShape<RB>::kThreads;
    static constexpr int kDPT = DIG / kDigitThreads;
    static constexpr int kDigitWarps = kDigitThreads / 32;
};

// One pass over the keys counts every digit position: hist[pass][DIG].  A few CTAs
// per SM each count a long stretch of keys into shared memory (16-byte loads, two in
// flight per thread), then add their counts to the global histogram once: with one
// CTA per few thousand keys, the global atomics of the flush (passes x DIG per CTA)
// cost more than the counting.
constexpr int kHistThreads = 512;
template <int RB>
__global__ void __launch_bounds__(kHistThreads) k_radix_histogram(const uint32_t* __restrict__ keys, int64_t n,
                                                                  int passes, uint32_t* __restrict__ hist) {
    using R = Radix<RB>;
    __shared__ uint32_t s_h[kHistWords];
    for (int i = threadIdx.x; i < passes * R::DIG; i += blockDim.x) s_h[i] = 0;
    __syncthreads();
    auto count = [&](uint32_t k) {
        for (int p = 0; p < passes; ++p) atomicAdd(&s_h[p * R::DIG + ((k >> (RB * p)) & R::MASK)], 1u);
    };
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t t0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    // 16-byte loads where the pointer allows them; the head before the first 16-byte
    // boundary and the tail after the last whole quad take single loads
    const int head = (int)((16 - ((uintptr_t)keys & 15)) & 15) / 4;
    const int64_t h = head < n ? head : n;
    const uint4* q = reinterpret_cast<const uint4*>(keys + h);
    const int64_t nq = ((uintptr_t)keys & 3) ? 0 : (n - h) / 4;
    int64_t i = t0;
    for (; i + stride < nq; i += 2 * stride) {
        const uint4 a = __ldg(q + i), b = __ldg(q + i + stride);
        count(a.x); count(a.y); count(a.z); count(a.w);
        count(b.x); count(b.y); count(b.z); count(b.w);
    }
    for (; i < nq; i += stride) {
        const uint4 a = __ldg(q + i);
        count(a.x); count(a.y); count(a.z); count(a.w);
    }
    const int64_t done = nq > 0 ? h + 4 * nq : 0;
    if (nq > 0)
        for (int64_t j = t0; j < h; j += stride) count(keys[j]);
    for (int64_t j = done + t0; j < n; j += stride) count(keys[j]);
    __syncthreads();
    for (int i2 = threadIdx.x; i2 < passes * R::DIG; i2 += blockDim.x) {
        const uint32_t c = s_h[i2];
        if (c) atomicAdd(&hist[i2], c);
    }
}

// One onesweep pass.  Warp w of a tile owns keys [w*32*IT, (w+1)*32*IT) of the tile
// in a warp-striped layout (item j of lane l is key j*32 + l), so processing items in
// order and lanes in order is index order: the ranks are stable.
template <int RB>
__global__ void __launch_bounds__(SortShape<RB>::kThreads, SortShape<RB>::kMinBlocks) k_onesweep(const uint32_t* __restrict__ kin,
                                                           const uint32_t* __restrict__ vin,
                                                           uint32_t* __restrict__ kout, uint32_t* __restrict__ vout,
                                                           int64_t n, int shift, const uint32_t* __restrict__ bins,
                                                           uint32_t* __restrict__ look, unsigned int* tile_counter,
                                                           int* err, uint32_t* __restrict__ cell_count,
                                                           uint32_t ncells) {
    using R = Radix<RB>;
    constexpr int kSortThreads = SortShape<RB>::kThreads;
    constexpr int kSortTile = SortShape<RB>::kTile;
    constexpr int kWarps = SortShape<RB>::kWarps;
    constexpr int DIG = R::DIG;
    constexpr int DPT = R::kDPT;
    // per warp and digit: the warp's count, then the tile-local position of the warp's
    // first key of that digit (at most 7680, so 16 bits)
    __shared__ uint16_t s_warp_hist[kWarps][DIG];
    __shared__ uint32_t s_count[DIG];        // the tile's count of each digit
    __shared__ uint32_t s_delta[DIG];        // global start minus tile-local start of each digit
    __shared__ uint32_t s_w[R::kDigitWarps];
    __shared__ uint32_t s_hw[R::kDigitWarps];
    extern __shared__ uint32_t s_staging[];  // keys, values in tile-sorted order [, values as loaded]
    uint32_t* s_keys = s_staging;
    uint32_t* s_vals = s_staging + kSortTile;
    uint32_t* s_vraw = s_vals;   // values as loaded, until the staging step
    __shared__ uint32_t s_tile;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) s_tile = atomicAdd(tile_counter, 1u);
    for (int i = threadIdx.x; i < kWarps * DIG / 2; i += kSortThreads)
        reinterpret_cast<uint32_t*>(&s_warp_hist[0][0])[i] = 0;
    for (int i = threadIdx.x; i < DIG; i += kSortThreads) s_count[i] = 0;
    // ranking: per warp and value of a digit's low 8 bits, the lanes holding it (in the
    // keys' staging area, which is free until the staging step)
    static_assert(kWarps * 256 <= kSortTile, "match words fit in the keys' staging area");
    uint32_t* s_match = s_staging;
    for (int i = threadIdx.x; i < kWarps * 256; i += kSortThreads) s_match[i] = 0;
    __syncthreads();
    const uint32_t tile = s_tile;
    const int64_t tbase = (int64_t)tile * kSortTile;
    const int64_t wbase = tbase + (int64_t)warp * 32 * kSortItems;
    // item j of this lane is in range iff j * 32 < rem
    const int64_t rem64 = n - (wbase + lane);
    const int rem = rem64 < kSortTile ? (int)rem64 : kSortTile;
    // values are not held in registers (fewer registers, more warps per SM): 8-bit passes
    // copy them into the values' area with cp.async while the tile ranks, 10-bit passes
    // read them at the staging step
    uint32_t key[kSortItems], rank[kSortItems];
#pragma unroll
    for (int j = 0; j < kSortItems; ++j) {
        const int64_t idx = wbase + j * 32 + lane;
        const bool ok = j * 32 < rem;
        key[j] = ok ? kin[idx] : 0xffffffffu;
        if constexpr (kValuePrefetch<RB>) {
            if (ok) {
                const uint32_t dst =
                    (uint32_t)__cvta_generic_to_shared(s_vraw + warp * 32 * kSortItems + j * 32 + lane);
                asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(dst), "l"(vin + idx) : "memory");
            }
        }
    }
    if constexpr (kValuePrefetch<RB>) asm volatile("cp.async.commit_group;\n" ::: "memory");
    // the tile's digit counts first (order-free shared-memory atomics), published
    // before the ranking so that the look-back of later tiles can start early
#pragma unroll
    for (int j = 0; j < kSortItems; ++j)
        if (j * 32 < rem) atomicAdd(&s_count[(key[j] >> shift) & R::MASK], 1u);
    __syncthreads();
    // digit thread t owns digits t*DPT .. t*DPT + DPT - 1
    const bool digit_thread = threadIdx.x < R::kDigitThreads;
    const int d0 = threadIdx.x * DPT;
    uint32_t tile_count[DPT];
    uint32_t* lk = look + (size_t)tile * DIG;
    // exclusive scan of the tile's counts over the digits (tile-local starts): the digit
    // warps' totals here, the scan itself after the ranking (the counts are re-read from
    // shared memory then, so nothing of this stays live across the ranking)
    const auto warp_scan = [&](uint32_t& mine) {
        mine = 0;
#pragma unroll
        for (int q = 0; q < DPT; ++q) {
            tile_count[q] = digit_thread ? s_count[d0 + q] : 0u;
            mine += tile_count[q];
        }
        uint32_t incl = mine;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        return incl;
    };
    if (digit_thread) {
        uint32_t mine;
        const uint32_t incl = warp_scan(mine);
        if (lane == 31) s_w[warp] = incl;
#pragma unroll
        for (int q = 0; q < DPT; ++q)
            if (tile > 0) st_relaxed_u32(&lk[d0 + q], kFlagA | tile_count[q]);
    }
    // tile 0 alone scans the pass's digit counts into the digits' global starts and
    // publishes start + its own count as its inclusive prefix, so every later tile's
    // look-back sum already holds its digit's global start
    if (tile == 0) {
        uint32_t hc[DPT], hmine = 0;
#pragma unroll
        for (int q = 0; q < DPT; ++q) {
            hc[q] = digit_thread ? bins[d0 + q] : 0u;
            hmine += hc[q];
        }
        uint32_t hincl = hmine;
        if (digit_thread) {
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t t = __shfl_up_sync(0xffffffffu, hincl, o);
                if (lane >= o) hincl += t;
            }
            if (lane == 31) s_hw[warp] = hincl;
        }
        __syncthreads();
        if (digit_thread) {
            uint32_t hoff = hincl - hmine;
            for (int w = 0; w < warp; ++w) hoff += s_hw[w];
#pragma unroll
            for (int q = 0; q < DPT; ++q) {
                st_relaxed_u32(&lk[d0 + q], kFlagP | ((hoff + tile_count[q]) & kValMask));
                s_delta[d0 + q] = hoff;   // this tile's exclusive prefix
                hoff += hc[q];
            }
        }
    }
    // warp-level ranking (stable): the lanes holding the same digit, as the lanes that
    // set their bit in the word of the digit's low 8 bits (shared-memory atomicOr) and,
    // for 10-bit digits, agree on the top bits by ballot
    const unsigned lt = (1u << lane) - 1u;
#pragma unroll
    for (int j = 0; j < kSortItems; ++j) {
        const bool ok = j * 32 < rem;
        const uint32_t dj = (key[j] >> shift) & R::MASK;
        uint32_t* m = s_match + warp * 256 + (dj & 255u);
        if (ok) atomicOr(m, 1u << lane);
        __syncwarp();
        const unsigned low = ok ? *m : 0u;
        __syncwarp();
        unsigned peers = low;
#pragma unroll
        for (int b = 8; b < RB; ++b) {
            const unsigned bal = __ballot_sync(0xffffffffu, (dj >> b) & 1u);
            peers &= ((dj >> b) & 1u) ? bal : ~bal;
        }
        // the lowest lane holding a low-8-bit value clears its word for the next item
        if (ok && lane == __ffs(low) - 1) *m = 0u;
        // the lowest lane of each group adds the group to the warp's digit count; the
        // count before it comes back to the whole group by one full-warp shuffle
        const int leader = peers ? __ffs(peers) - 1 : lane;
        uint32_t prior = 0;
        if (ok && lane == leader) {
            prior = s_warp_hist[warp][dj];
            s_warp_hist[warp][dj] = (uint16_t)(prior + __popc(peers));
        }
        prior = __shfl_sync(0xffffffffu, prior, leader);
        rank[j] = prior + __popc(peers & lt);
        __syncwarp();
    }
    __syncthreads();
    // per digit: tile-local start, then the start of each warp's keys of that digit (in
    // place of the warp's count)
    uint32_t toff[DPT], excl[DPT];
    if (digit_thread) {
        uint32_t mine;
        uint32_t o = warp_scan(mine) - mine;
        for (int w = 0; w < warp; ++w) o += s_w[w];
#pragma unroll
        for (int q = 0; q < DPT; ++q) {
            toff[q] = o;
            uint32_t run = o;
#pragma unroll
            for (int w = 0; w < kWarps; ++w) {
                const uint32_t c = s_warp_hist[w][d0 + q];
                s_warp_hist[w][d0 + q] = (uint16_t)run;
                run += c;
            }
            o += tile_count[q];
        }
    }
    // look back for the prefix of each owned digit: kLookWindow tiles at a time (the
    // loads of all owned digits in flight together), summing the counts up to and
    // including the nearest inclusive prefix (tile 0's holds the digit's global start)
#pragma unroll
    for (int q = 0; q < DPT; ++q) excl[q] = (digit_thread && tile == 0) ? s_delta[d0 + q] : 0u;
    if (digit_thread && tile > 0) {
        bool done[DPT];
#pragma unroll
        for (int q = 0; q < DPT; ++q) done[q] = false;
        int64_t t = (int64_t)tile - 1;
        uint32_t spins = 0;
        while (true) {
            bool all_done = true;
#pragma unroll
            for (int q = 0; q < DPT; ++q) all_done = all_done && done[q];
            if (all_done) break;
            uint32_t w[DPT][kLookWindow];
#pragma unroll
            for (int q = 0; q < DPT; ++q)
#pragma unroll
                for (int j = 0; j < kLookWindow; ++j)
                    w[q][j] = (!done[q] && t - j >= 0) ? ld_relaxed_u32(&look[(size_t)(t - j) * DIG + d0 + q]) : kFlagP;
            bool ready = true;
#pragma unroll
            for (int q = 0; q < DPT; ++q)
#pragma unroll
                for (int j = 0; j < kLookWindow; ++j) ready = ready && (w[q][j] & ~kValMask) != 0;
            if (!ready) {
                if (++spins > kSpinLimit) {
                    atomicExch(err, 1);
                    break;
                }
                continue;
            }
#pragma unroll
            for (int q = 0; q < DPT; ++q) {
#pragma unroll
                for (int j = 0; j < kLookWindow; ++j) {
                    if (!done[q]) {
                        excl[q] += w[q][j] & kValMask;
                        done[q] = (w[q][j] & ~kValMask) == kFlagP;
                    }
                }
            }
            t -= kLookWindow;
        }
#pragma unroll
        for (int q = 0; q < DPT; ++q) st_relaxed_u32(&lk[d0 + q], kFlagP | ((excl[q] + tile_count[q]) & kValMask));
    }
    if (digit_thread) {
#pragma unroll
        for (int q = 0; q < DPT; ++q) s_delta[d0 + q] = excl[q] - toff[q];
    }
    // each thread reads back only the values it copied itself, so its own wait suffices
    if constexpr (kValuePrefetch<RB>) asm volatile("cp.async.wait_all;\n" ::: "memory");
    __syncthreads();
    if constexpr (kValuePrefetch<RB>) {
        // stage keys in tile-sorted order, taking each thread's values out of the values'
        // area (into the keys' registers) and their positions (into the ranks' registers)
#pragma unroll
        for (int j = 0; j < kSortItems; ++j) {
            if (j * 32 < rem) {
                const uint32_t dd = (key[j] >> shift) & R::MASK;
                const uint32_t lp = s_warp_hist[warp][dd] + rank[j];
                s_keys[lp] = key[j];
                rank[j] = lp;
                key[j] = s_vraw[warp * 32 * kSortItems + j * 32 + lane];
            }
        }
        __syncthreads();
        // then the values
#pragma unroll
        for (int j = 0; j < kSortItems; ++j)
            if (j * 32 < rem) s_vals[rank[j]] = key[j];
    } else {
        // stage keys and values in tile-sorted order
#pragma unroll
        for (int j = 0; j < kSortItems; ++j) {
            if (j * 32 < rem) {
                const uint32_t dd = (key[j] >> shift) & R::MASK;
                const uint32_t lp = s_warp_hist[warp][dd] + rank[j];
                s_keys[lp] = key[j];
                s_vals[lp] = vin[wbase + j * 32 + lane];
            }
        }
    }
    __syncthreads();
    const int valid = (int)(n - tbase < kSortTile ? n - tbase : kSortTile);
    if (!cell_count) {
        for (int i = threadIdx.x; i < valid; i += kSortThreads) {
            const uint32_t k = s_keys[i];
            const uint32_t g = s_delta[(k >> shift) & R::MASK] + (uint32_t)i;
            kout[g] = k;
            vout[g] = s_vals[i];
        }
        return;
    }
    // last pass with cell counts: the staged keys are the tile's keys in full order, so
    // a warp's 32 consecutive keys form a few runs of equal cells; the last lane of each
    // run adds the run's length (whole warps step together for the shuffles)
    for (int b = threadIdx.x - lane; b < valid; b += kSortThreads) {
        const int i = b + lane;
        const bool ok = i < valid;
        const uint32_t k = ok ? s_keys[i] : 0xffffffffu;
        if (ok) {
            const uint32_t g = s_delta[(k >> shift) & R::MASK] + (uint32_t)i;
            kout[g] = k;
            vout[g] = s_vals[i];
        }
        const uint32_t prev = __shfl_up_sync(0xffffffffu, k, 1);
        const uint32_t next = __shfl_down_sync(0xffffffffu, k, 1);
        const unsigned starts = __ballot_sync(0xffffffffu, lane == 0 || k != prev);
        if (ok && k < ncells && (lane == 31 || k != next)) {
            const int first = 31 - __clz(starts & (0xffffffffu >> (31 - lane)));
            atomicAdd(&cell_count[k], (uint32_t)(lane - first + 1));
        }
    }
}

// Counts per cell.  Equal neighbours within a warp are added as one run (the keys come
// sorted, so a warp holds a few runs): the last lane of each run adds its length.
__global__ void k_histogram_cells(const uint32_t* __restrict__ keys, int64_t n, uint32_t ncells,
                                  uint32_t* __restrict__ count) {
    const int lane = threadIdx.x & 31;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t base = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) - lane; base < n; base += stride) {
        const int64_t i = base + lane;
        const uint32_t k = i < n ? keys[i] : 0xffffffffu;   // past the end: no cell
        const uint32_t prev = __shfl_up_sync(0xffffffffu, k, 1);
        const uint32_t next = __shfl_down_sync(0xffffffffu, k, 1);
        const unsigned starts = __ballot_sync(0xffffffffu, lane == 0 || k != prev);
        const bool last = lane == 31 || k != next;
        if (last && k < ncells) {
            const int first = 31 - __clz(starts & (0xffffffffu >> (31 - lane)));
            atomicAdd(&count[k], (uint32_t)(lane - first + 1));
        }
    }
}

__global__ void k_left_right(const uint32_t* __restrict__ start, const uint32_t* __restrict__ count, int64_t ncells,
                             uint32_t* __restrict__ left, uint32_t* __restrict__ right) {
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < ncells;
         c += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t s = start[c], k = count[c];
        left[c] = s;
        right[c] = k ? s + k - 1 : s;
    }
}

inline unsigned grid_cap(int64_t n, int threads) {
    int64_t b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > 148 * 16) b = 148 * 16;
    return (unsigned)b;
}

inline size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

}  // namespace

size_t scan_scratch_bytes(int64_t n) {
    const int64_t tiles = (n + kScanTile - 1) / kScanTile;
    return (size_t)(2 + tiles) * sizeof(uint64_t);
}

cudaError_t scan_exclusive_u32(const uint32_t* in, uint32_t* out, int64_t n, void* scratch, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    const int64_t tiles = (n + kScanTile - 1) / kScanTile;
    cudaError_t e = cudaMemsetAsync(scratch, 0, scan_scratch_bytes(n), st);
    if (e != cudaSuccess) return e;
    const int vec = (((uintptr_t)in | (uintptr_t)out) & 15u) == 0 ? 1 : 0;
    const int smem = (int)(sizeof(uint4) * (kScanQuads + kScanQuads / 8));
    e = cudaFuncSetAttribute(k_scan_exclusive, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    k_scan_exclusive<<<(unsigned)tiles, kScanThreads, smem, st>>>(in, out, n, (uint64_t*)scratch, vec);
    return cudaGetLastError();
}

int scan_error_flag_offset() { return 8; }   // byte offset of the error word inside the scan scratch

SortLayout sort_layout(int64_t n, int key_bits) {
    SortLayout L{};
    if (key_bits < 1) key_bits = 1;
    if (key_bits > 32) key_bits = 32;
    const int p8 = (key_bits + 7) / 8, p10 = (key_bits + 9) / 10;
    // 10-bit digits where they save a pass (17-20 and 25-30 key bits)
    L.digit_bits = (key_bits > 16 && key_bits <= 30 && p10 < p8) ? 10 : 8;
    L.passes = L.digit_bits == 10 ? p10 : p8;
    const int tile = L.digit_bits == 10 ? SortShape<10>::kTile : SortShape<8>::kTile;
    L.tiles = (n + tile - 1) / tile;
    size_t off = 0;
    L.off_hist = off;    off += align256(sizeof(uint32_t) * kHistWords);
    L.off_counters = off; off += align256(sizeof(uint32_t) * 8);     // tile counters [4], error word [4]
    // look-back words for the widest layout (4 passes x 256 digits x 3840-key tiles, or
    // 3 x 1024 x 7680-key tiles), so that the scratch size does not depend on key_bits
    const int64_t t8 = (n + SortShape<8>::kTile - 1) / SortShape<8>::kTile;
    const int64_t t10 = (n + SortShape<10>::kTile - 1) / SortShape<10>::kTile;
    const int64_t look_words = std::max<int64_t>(std::max<int64_t>(4 * 256 * t8, 3 * 1024 * t10), 3 * 1024);
    L.off_look = off;    off += align256(sizeof(uint32_t) * (size_t)look_words);
    L.off_alt_keys = off; off += align256(sizeof(uint32_t) * (size_t)(n > 0 ? n : 1));
    L.off_alt_vals = off; off += align256(sizeof(uint32_t) * (size_t)(n > 0 ? n : 1));
    L.bytes = off;
    return L;
}

cudaError_t radix_sort_begin(int64_t n, int key_bits, void* scratch, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    const SortLayout L = sort_layout(n, key_bits);
    cudaError_t e = L.digit_bits == 10
                        ? cudaFuncSetAttribute(k_onesweep<10>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               SortShape<10>::kStagingBytes)
                        : cudaFuncSetAttribute(k_onesweep<8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               SortShape<8>::kStagingBytes);
    if (e != cudaSuccess) return e;
    return cudaMemsetAsync(scratch, 0,
                           L.off_look + sizeof(uint32_t) * ((size_t)1 << L.digit_bits) * (size_t)L.tiles * L.passes, st);
}

uint32_t* radix_sort_hist(int64_t n, int key_bits, void* scratch) {
    return (uint32_t*)((char*)scratch + sort_layout(n, key_bits).off_hist);
}

cudaError_t radix_sort_finish(const uint32_t* kin, const uint32_t* vin, uint32_t* kout, uint32_t* vout, int64_t n,
                              int key_bits, void* scratch, cudaStream_t st, uint32_t* cell_count, int64_t ncells) {
    if (n <= 0) return cudaSuccess;
    const SortLayout L = sort_layout(n, key_bits);
    const int rb = L.digit_bits, dig = 1 << rb;
    char* base = (char*)scratch;
    uint32_t* hist = (uint32_t*)(base + L.off_hist);
    uint32_t* counters = (uint32_t*)(base + L.off_counters);
    uint32_t* look = (uint32_t*)(base + L.off_look);
    uint32_t* ak = (uint32_t*)(base + L.off_alt_keys);
    uint32_t* av = (uint32_t*)(base + L.off_alt_vals);
    // ping-pong so that the last pass lands in (kout, vout)
    const uint32_t* sk = kin;
    const uint32_t* sv = vin;
    for (int p = 0; p < L.passes; ++p) {
        const bool to_out = ((L.passes - 1 - p) % 2) == 0;
        uint32_t* dk = to_out ? kout : ak;
        uint32_t* dv = to_out ? vout : av;
        uint32_t* lp = look + (size_t)dig * L.tiles * p;
        uint32_t* cc = p == L.passes - 1 ? cell_count : nullptr;
        if (rb == 10)
            k_onesweep<10><<<(unsigned)L.tiles, SortShape<10>::kThreads, SortShape<10>::kStagingBytes, st>>>(
                sk, sv, dk, dv, n, rb * p, hist + dig * p, lp, counters + p, (int*)(counters + 4), cc,
                (uint32_t)ncells);
        else
            k_onesweep<8><<<(unsigned)L.tiles, SortShape<8>::kThreads, SortShape<8>::kStagingBytes, st>>>(
                sk, sv, dk, dv, n, rb * p, hist + dig * p, lp, counters + p, (int*)(counters + 4), cc,
                (uint32_t)ncells);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        sk = dk;
        sv = dv;
    }
    return cudaSuccess;
}

cudaError_t radix_sort_pairs_u32(const uint32_t* kin, const uint32_t* vin, uint32_t* kout, uint32_t* vout, int64_t n,
                                 int key_bits, void* scratch, cudaStream_t st, uint32_t* cell_count, int64_t ncells) {
    if (n <= 0) return cudaSuccess;
    cudaError_t e = radix_sort_begin(n, key_bits, scratch, st);
    if (e != cudaSuccess) return e;
    const SortLayout L = sort_layout(n, key_bits);
    uint32_t* hist = radix_sort_hist(n, key_bits, scratch);
    // about 16 keys per thread, at most two CTAs per SM
    int64_t hb = (n + (int64_t)kHistThreads * 16 - 1) / ((int64_t)kHistThreads * 16);
    if (hb < 1) hb = 1;
    if (hb > 148 * 2) hb = 148 * 2;
    if (L.digit_bits == 10) k_radix_histogram<10><<<(unsigned)hb, kHistThreads, 0, st>>>(kin, n, L.passes, hist);
    else k_radix_histogram<8><<<(unsigned)hb, kHistThreads, 0, st>>>(kin, n, L.passes, hist);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    return radix_sort_finish(kin, vin, kout, vout, n, key_bits, scratch, st, cell_count, ncells);
}

cudaError_t cell_counts_u32(const uint32_t* sorted_keys, int64_t n, int64_t ncells, uint32_t* count, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(count, 0, sizeof(uint32_t) * (size_t)ncells, st);
    if (e != cudaSuccess) return e;
    if (n > 0) k_histogram_cells<<<grid_cap(n, 256), 256, 0, st>>>(sorted_keys, n, (uint32_t)ncells, count);
    return cudaGetLastError();
}

cudaError_t cell_offsets_u32(const uint32_t* sorted_keys, int64_t n, int64_t ncells, uint32_t* start, uint32_t* count,
                             void* scan_scratch, cudaStream_t st) {
    cudaError_t e = cell_counts_u32(sorted_keys, n, ncells, count, st);
    if (e != cudaSuccess) return e;
    return scan_exclusive_u32(count, start, ncells, scan_scratch, st);
}

cudaError_t left_right_u32(const uint32_t* start, const uint32_t* count, int64_t ncells, uint32_t* left,
                           uint32_t* right, cudaStream_t st) {
    k_left_right<<<grid_cap(ncells, 256), 256, 0, st>>>(start, count, ncells, left, right);
    return cudaGetLastError();
}

}  // namespace gpgmp

// ---- exclusive scan without allocation -----------------------------------------
// For callers that must not call cudaMalloc: the scan's scratch (tile counter,
// error word, one status word per 16384-value tile) lives in a fixed file-scope
// device array instead of a caller buffer.  Every device that loads this library
// holds the array (32 KiB) until the process exits; it serves scans of up to
// kNoAllocMaxN values.
namespace gpgmp {
namespace {
constexpr int64_t kNoAllocMaxN = (int64_t)1 << 26;
constexpr size_t kNoAllocWords = 2 + (size_t)(kNoAllocMaxN / kScanTile);
static __device__ __align__(256) uint64_t g_noalloc_scan_scratch[kNoAllocWords];

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mu;
void* g_noalloc_addr[kNoAllocMaxDevices] = {};

// Device address of the array on the current device.  In host code the array's
// name only stands in for the symbol, so the address comes from
// cudaGetSymbolAddress, once per device, with that device current.
int noalloc_scratch(void** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return set_error(GPGMP_ERR_CUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
    if (dev < 0 || dev >= kNoAllocMaxDevices) return set_error(GPGMP_ERR_UNSUPPORTED, "device %d", dev);
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scan_scratch);
        if (e != cudaSuccess || !p)
            return set_error(GPGMP_ERR_CUDA, "cudaGetSymbolAddress: %s", cudaGetErrorString(e));
        g_noalloc_addr[dev] = p;
    }
    *out = g_noalloc_addr[dev];
    return GPGMP_OK;
}
}  // namespace
}  // namespace gpgmp

extern "C" int gpgmp_exclusive_scan_u32_noalloc(const uint32_t* in, uint32_t* out, int64_t n, void* stream) {
    using namespace gpgmp;
    if (n < 0 || (n > 0 && (!in || !out))) return set_error(GPGMP_ERR_INVALID, "bad argument");
    if (n > kNoAllocMaxN)
        return set_error(GPGMP_ERR_INVALID, "n = %lld exceeds the %lld values the built-in scratch serves",
                         (long long)n, (long long)kNoAllocMaxN);
    if (n == 0) return GPGMP_OK;
    void* scratch = nullptr;
    int rc = noalloc_scratch(&scratch);
    if (rc) return rc;
    // zeroes the counter, the error word and the status words this scan uses, then scans
    cudaError_t e = scan_exclusive_u32(in, out, n, scratch, (cudaStream_t)stream);
    if (e != cudaSuccess) return set_error(GPGMP_ERR_CUDA, "scan: %s", cudaGetErrorString(e));
    return GPGMP_OK;
}

// Waits for `stream` and reads the error word of the built-in scratch: GPGMP_ERR_TIMEOUT
// in *status when the last scan's look-back gave up (its output is then wrong).  The
// next no-allocation scan clears the word, so this is read before it.
extern "C" int gpgmp_exclusive_scan_u32_noalloc_status(void* stream, int32_t* status) {
    using namespace gpgmp;
    if (!status) return set_error(GPGMP_ERR_INVALID, "bad argument");
    void* scratch = nullptr;
    int rc = noalloc_scratch(&scratch);
    if (rc) return rc;
    cudaError_t e = cudaStreamSynchronize((cudaStream_t)stream);
    if (e != cudaSuccess) return set_error(GPGMP_ERR_CUDA, "cudaStreamSynchronize: %s", cudaGetErrorString(e));
    uint32_t word = 0;
    e = cudaMemcpy(&word, (const char*)scratch + scan_error_flag_offset(), sizeof(word), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return set_error(GPGMP_ERR_CUDA, "cudaMemcpy: %s", cudaGetErrorString(e));
    *status = word ? GPGMP_ERR_TIMEOUT : GPGMP_OK;
    return GPGMP_OK;
}
