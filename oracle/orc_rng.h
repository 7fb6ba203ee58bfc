/*
 * oracle/orc_rng.h -- TEST INFRASTRUCTURE ONLY (the oracle).
 *
 * CPU restatements of the two counter-based generators used on the hot path:
 *
 *  - Threefry-2x32-20, the generator the reference's OpenCL kernels draw from
 *    (reference: exec/src/gpgmp/src/cl_include/Random123/threefry.h:135-142 rotation
 *    table, :172 key-schedule parity, :733 default 20 rounds; used at
 *    Gillespie.cl:41-42, StochasticHomogeneousDiffusion.cl:19-20,
 *    StochasticInhomogeneousDriftDiffusion.cl:448-452).
 *  - Philox-4x32-10, the generator the CUDA kernels of this project draw from.
 *
 * Both are written from the published description (Salmon, Moraes, Dror, Shaw,
 * "Parallel random numbers: as easy as 1, 2, 3", SC'11).  They are pinned against
 * the reference's vendored Random123 headers by tests/test_oracle_pin.py, which
 * compiles those headers into oracle/_ref.
 *
 * Nothing in the product may include this file.
 */
#ifndef ORC_RNG_H
#define ORC_RNG_H
#include <stdint.h>

static inline uint32_t orc_rotl32(uint32_t x, unsigned n) {
    n &= 31u;
    return n ? (uint32_t)((x << n) | (x >> (32u - n))) : x;
}

/* Threefry-2x32 with 20 rounds: 4-round groups, key injected after each group. */
static inline void orc_threefry2x32_20_inl(const uint32_t ctr[2], const uint32_t key[2], uint32_t out[2]) {
    static const unsigned rot[8] = {13, 15, 26, 6, 17, 29, 16, 24};
    uint32_t ks[3];
    ks[0] = key[0];
    ks[1] = key[1];
    ks[2] = 0x1BD11BDAu ^ key[0] ^ key[1];
    uint32_t x0 = ctr[0] + ks[0];
    uint32_t x1 = ctr[1] + ks[1];
    for (unsigned r = 0; r < 20; ++r) {
        x0 += x1;
        x1 = orc_rotl32(x1, rot[r & 7u]);
        x1 ^= x0;
        if ((r & 3u) == 3u) {
            unsigned s = (r >> 2) + 1u; /* injection number 1..5 */
            x0 += ks[s % 3u];
            x1 += ks[(s + 1u) % 3u] + s;
        }
    }
    out[0] = x0;
    out[1] = x1;
}

/* Philox-4x32 with 10 rounds. */
static inline void orc_philox4x32_10_inl(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    uint32_t x0 = ctr[0], x1 = ctr[1], x2 = ctr[2], x3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)0xD2511F53u * x0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * x2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        x0 = hi1 ^ x1 ^ k0;
        x1 = lo1;
        x2 = hi0 ^ x3 ^ k1;
        x3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = x0; out[1] = x1; out[2] = x2; out[3] = x3;
}

/* A Philox stream: fixed key, counter word 0 walks, 4 outputs buffered. */
typedef struct {
    uint32_t key[2];
    uint32_t ctr[4];
    uint32_t buf[4];
    int idx;
} orc_stream;

static inline void orc_stream_init(orc_stream* s, uint32_t k0, uint32_t k1,
                                   uint32_t c1, uint32_t c2, uint32_t c3) {
    s->key[0] = k0; s->key[1] = k1;
    s->ctr[0] = 0; s->ctr[1] = c1; s->ctr[2] = c2; s->ctr[3] = c3;
    s->idx = 4;
}

static inline uint32_t orc_stream_next(orc_stream* s) {
    if (s->idx == 4) {
        orc_philox4x32_10_inl(s->ctr, s->key, s->buf);
        s->ctr[0] += 1u;
        s->idx = 0;
    }
    return s->buf[s->idx++];
}

/* Stream phase tags (counter word 3, top byte); low bits carry species/sweep. */
#define ORC_PH_INIT   0x01000000u
#define ORC_PH_SSA    0x02000000u
#define ORC_PH_DIFF   0x03000000u
#define ORC_PH_SOURCE 0x04000000u
#define ORC_PH_PART   0x05000000u
#define ORC_PH_PAIR   0x06000000u
#define ORC_PH_POP    0x07000000u
#define ORC_PH_INDIV  0x08000000u
#define ORC_PH_NEWIND 0x09000000u

#endif
