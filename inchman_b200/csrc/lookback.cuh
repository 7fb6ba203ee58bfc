// Decoupled look-back (Merrill & Garland 2016, "Single-pass Parallel Prefix Scan
// with Decoupled Look-back"): the tile-status words and the warp-wide look-back
// shared by the single-pass scans of sort.cu and population.cu.
//
// A tile status word is (flag << 32) | value: flag 0 = not yet published, 1 = the
// tile's own aggregate, 2 = the inclusive prefix up to and including the tile.
// Tiles take their index from an atomic counter in launch order, so a tile only
// waits for tiles that are already running; the wait still has an iteration limit,
// after which the error word is set and the tile carries on with what it has.
#pragma once
#include <cstdint>

namespace gpgmp {

constexpr uint64_t kScanFlagA = 1ull << 32;
constexpr uint64_t kScanFlagP = 2ull << 32;
constexpr uint32_t kSpinLimit = 1u << 24;

__device__ __forceinline__ uint64_t ld_volatile_u64(const uint64_t* p) {
    uint64_t v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];\n" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_u64(uint64_t* p, uint64_t v) {
    asm volatile("st.release.gpu.global.u64 [%0], %1;\n" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ void st_relaxed_u64(uint64_t* p, uint64_t v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;\n" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ uint32_t ld_acquire_u32(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_u32(uint32_t* p, uint32_t v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;\n" ::"l"(p), "r"(v) : "memory");
}
// For status words that carry their whole payload (flag and value in one word, no
// other data published with them) relaxed accesses suffice: no fence per access.
__device__ __forceinline__ uint32_t ld_relaxed_u32(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed_u32(uint32_t* p, uint32_t v) {
    asm volatile("st.relaxed.gpu.global.u32 [%0], %1;\n" ::"l"(p), "r"(v) : "memory");
}

constexpr int kLookDepth = 4;   // status words per lane per round: 128 tiles

// Called by all 32 lanes of one warp.  Publishes tile's aggregate, looks back over
// the preceding tiles 128 at a time (lane l, slot u reads the tile 32 u + l + 1
// before the window's start, so the nearest tiles come first), publishes the
// inclusive prefix and returns the exclusive prefix (in every lane).  Only the tiles
// up to the nearest one with an inclusive prefix need to have published; the loads
// of a round are independent, so a tile far from any inclusive prefix sums 128
// aggregates per memory round trip.  A status word carries its whole payload (flag
// and value), so it is published and read with relaxed accesses (no fences).  err is
// set when a wait exceeds kSpinLimit.
__device__ __forceinline__ uint32_t warp_lookback_u32(uint64_t* status, uint32_t tile, uint32_t aggregate, int* err) {
    const int lane = threadIdx.x & 31;
    if (tile == 0) {
        if (lane == 0) st_relaxed_u64(&status[0], kScanFlagP | aggregate);
        return 0u;
    }
    if (lane == 0) st_relaxed_u64(&status[tile], kScanFlagA | aggregate);
    int64_t look = (int64_t)tile - 1;
    uint32_t exclusive = 0, spins = 0;
    while (true) {
        uint64_t w[kLookDepth];
#pragma unroll
        for (int u = 0; u < kLookDepth; ++u) {
            const int64_t idx = look - lane - 32 * u;
            w[u] = idx >= 0 ? ld_volatile_u64(&status[idx]) : kScanFlagP;   // before tile 0: prefix 0
        }
        // the nearest inclusive prefix of the round: slot pu, lane pl
        int pu = kLookDepth, pl = 31;
#pragma unroll
        for (int u = kLookDepth - 1; u >= 0; --u) {
            const unsigned m = __ballot_sync(0xffffffffu, (uint32_t)(w[u] >> 32) == 2u);
            if (m) {
                pu = u;
                pl = __ffs(m) - 1;
            }
        }
        // the tiles that count: every slot before pu, slot pu up to lane pl
        bool missing = false;
        uint32_t val = 0;
#pragma unroll
        for (int u = 0; u < kLookDepth; ++u) {
            if (u < pu || (u == pu && lane <= pl)) {
                missing |= (uint32_t)(w[u] >> 32) == 0u;
                val += (uint32_t)w[u];
            }
        }
        if (__any_sync(0xffffffffu, missing)) {
            if (++spins > kSpinLimit) {
                if (lane == 0) atomicExch(err, 1);
                break;
            }
            continue;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) val += __shfl_xor_sync(0xffffffffu, val, o);
        exclusive += val;
        if (pu < kLookDepth) break;
        look -= 32 * kLookDepth;
    }
    if (lane == 0) st_relaxed_u64(&status[tile], kScanFlagP | (uint32_t)(exclusive + aggregate));
    return exclusive;
}

}  // namespace gpgmp
