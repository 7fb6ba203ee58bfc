/*
 * oracle/orc_sort.c -- TEST INFRASTRUCTURE ONLY (the oracle).
 *
 * Sort, scan and cell-offset oracles for the individual-particle path, and a CPU
 * replay of the particle-binning step.
 *  - orc_sort_pairs_u32: stable sort of (key, value) by key, the result of the
 *    reference's LSD radix sort (IndividualSolver.cpp:673-757, kernels
 *    IndividualSolver.cl:36-369), i.e. std::stable_sort on the low 32 bits.
 *  - orc_exclusive_scan_u32: exclusive prefix sum modulo 2^32
 *    (IndividualSolver.cl:493-553, IndividualSolver.cpp:759-808).
 *  - orc_cell_indices_ref: literal restatement of computeCellIndices
 *    (IndividualSolver.cl:564-619, host IndividualSolver.cpp:1083-1098).
 *  - orc_cell_offsets: per-cell start (exclusive scan of the key histogram) and count.
 *  - orc_particles_run: replay of the binning step (Brownian move, sort, offsets,
 *    in-cell A+B->0 pairing, compaction).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "gpgmp_oracle.h"
#include "orc_math.h"

void orc_sort_pairs_u32(uint32_t* keys, uint32_t* vals, int64_t n) {
    if (n <= 1) return;
    uint32_t* k2 = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)n);
    uint32_t* v2 = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)n);
    uint32_t *ka = keys, *va = vals, *kb = k2, *vb = v2;
    for (int pass = 0; pass < 4; ++pass) {
        const int sh = 8 * pass;
        size_t cnt[257];
        memset(cnt, 0, sizeof cnt);
        for (int64_t i = 0; i < n; ++i) cnt[((ka[i] >> sh) & 0xffu) + 1]++;
        for (int b = 0; b < 256; ++b) cnt[b + 1] += cnt[b];
        for (int64_t i = 0; i < n; ++i) {
            size_t d = cnt[(ka[i] >> sh) & 0xffu]++;
            kb[d] = ka[i];
            vb[d] = va[i];
        }
        uint32_t* t;
        t = ka; ka = kb; kb = t;
        t = va; va = vb; vb = t;
    }
    /* four passes: data is back in the caller's arrays */
    free(k2); free(v2);
}

void orc_exclusive_scan_u32(const uint32_t* in, uint32_t* out, int64_t n) {
    uint32_t acc = 0;
    for (int64_t i = 0; i < n; ++i) { uint32_t v = in[i]; out[i] = acc; acc += v; }
}

void orc_cell_indices_ref(const uint32_t* keys, int64_t nkeys, int64_t ncells, uint32_t* left, uint32_t* right) {
    if (nkeys <= 0) return;
    for (int64_t tid = 0; tid < nkeys; ++tid) {
        uint32_t myKey = keys[tid];
        if (tid == 0) {
            for (uint32_t i = 0; i < myKey; ++i) { left[i] = 0; right[i] = 0; }
            left[myKey] = 0;
        }
        if (tid < nkeys - 1) {
            uint32_t rightKey = keys[tid + 1];
            if (rightKey > myKey) {
                right[myKey] = (uint32_t)tid;
                for (uint32_t i = 1; i < rightKey - myKey; ++i) {
                    left[myKey + i] = (uint32_t)tid + 1;
                    right[myKey + i] = (uint32_t)tid + 1;
                }
                left[rightKey] = (uint32_t)tid + 1;
            }
        }
        if (tid == nkeys - 1) {
            right[myKey] = (uint32_t)tid;
            for (int64_t i = 1; i < ncells - (int64_t)myKey; ++i) {
                left[myKey + i] = (uint32_t)tid + 1;
                right[myKey + i] = (uint32_t)tid + 1;
            }
        }
    }
}

void orc_cell_offsets(const uint32_t* keys, int64_t n, int64_t ncells, uint32_t* start, uint32_t* count) {
    memset(count, 0, sizeof(uint32_t) * (size_t)ncells);
    for (int64_t i = 0; i < n; ++i) if (keys[i] < (uint64_t)ncells) count[keys[i]]++;
    orc_exclusive_scan_u32(count, start, ncells);
}

static inline float reflect_into(float x, float L) {
    if (x < 0.0f) x = -x;
    if (x >= L) x = (L + L) - x;
    if (x < 0.0f) x = 0.0f;
    if (x >= L) x = nextafterf(L, 0.0f);
    return x;
}

int64_t orc_particles_run(int64_t n, float* px, float* py, uint8_t* sp, int G, float D, float vx, float vy,
                          float dt, float p_react, uint32_t seed, int step0, int nsteps) {
    const float L = (float)G;
    const float sig = sqrtf(2.0f * D * dt);
    const float ax = vx * dt, ay = vy * dt;
    const int64_t ncells = (int64_t)G * G;
    /* floor(p 2^32), held to 2^32 - 1 for p = 1 (the largest 32-bit threshold) */
    const double tp = floor((double)p_react * 4294967296.0);
    const uint32_t thresh = tp < 4294967295.0 ? (uint32_t)tp : 4294967295u;
    uint32_t* keys = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)(n > 0 ? n : 1));
    uint32_t* vals = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)(n > 0 ? n : 1));
    uint32_t* start = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)ncells);
    uint32_t* count = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)ncells);
    uint8_t* alive = (uint8_t*)malloc((size_t)(n > 0 ? n : 1));
    float* nx = (float*)malloc(sizeof(float) * (size_t)(n > 0 ? n : 1));
    float* ny = (float*)malloc(sizeof(float) * (size_t)(n > 0 ? n : 1));
    uint8_t* nsp = (uint8_t*)malloc((size_t)(n > 0 ? n : 1));
    for (int k = step0; k < step0 + nsteps; ++k) {
        #pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; ++i) {
            orc_stream st;
            orc_stream_init(&st, seed, 0u, (uint32_t)k, (uint32_t)i, ORC_PH_PART);
            float z0, z1;
            orc_normal2(&st, &z0, &z1);
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
        orc_sort_pairs_u32(keys, vals, n);
        orc_cell_offsets(keys, n, ncells, start, count);
        memset(alive, 1, (size_t)n);
        #pragma omp parallel for schedule(dynamic, 1024)
        for (int64_t c = 0; c < ncells; ++c) {
            uint32_t s0 = start[c], cnt = count[c];
            if (cnt < 2) continue;
            orc_stream st;
            orc_stream_init(&st, seed, 1u, (uint32_t)k, (uint32_t)c, ORC_PH_PAIR);
            uint32_t ia = s0, ib = s0;
            const uint32_t e = s0 + cnt;
            for (;;) {
                while (ia < e && sp[vals[ia]] != 0) ia++;
                while (ib < e && sp[vals[ib]] != 1) ib++;
                if (ia >= e || ib >= e) break;
                uint32_t u = orc_stream_next(&st);
                if (u < thresh) { alive[ia] = 0; alive[ib] = 0; }
                ia++; ib++;
            }
        }
        int64_t m = 0;
        for (int64_t j = 0; j < n; ++j) {
            if (!alive[j]) continue;
            uint32_t src = vals[j];
            nx[m] = px[src]; ny[m] = py[src]; nsp[m] = sp[src];
            m++;
        }
        memcpy(px, nx, sizeof(float) * (size_t)m);
        memcpy(py, ny, sizeof(float) * (size_t)m);
        memcpy(sp, nsp, (size_t)m);
        n = m;
    }
    free(keys); free(vals); free(start); free(count); free(alive); free(nx); free(ny); free(nsp);
    return n;
}

/* IndividualSolver::maintainPopulation (IndividualSolver.cpp:458-671,
 * IndividualSolver.cl:1017-1882), restated as the CUDA path lays it out: per cell the
 * surplus is chosen by selection sampling (candidate i taken with probability
 * k_rem / (is - i): draw x, taken iff x (is - i) < k_rem 2^32; one Philox draw per
 * candidate while removals remain, stream (seed, 0, step, cell, POP)); the new
 * list has, per cell in order, the births (ids from the front of the pool) and then
 * the survivors in their old order; the new pool is the removed ids in list order
 * followed by the unused old pool.  Returns -1 if the pool is too small. */
int orc_population_maintain(const uint32_t* keys, const uint32_t* ids, int64_t n, const uint32_t* start,
                            const uint32_t* count, const int32_t* goal, int64_t ncells, const uint32_t* pool,
                            int64_t npool, uint32_t seed, uint32_t step, uint32_t* keys_out, uint32_t* ids_out,
                            uint32_t* pool_out, int64_t* n_out, int64_t* npool_out) {
    uint8_t* dead = (uint8_t*)calloc(n > 0 ? n : 1, 1);
    int64_t births = 0;
    for (int64_t c = 0; c < ncells; ++c) {
        uint32_t is = count[c], g = goal[c] > 0 ? (uint32_t)goal[c] : 0u;
        if (g > is) births += g - is;
        if (is > g) {
            orc_stream st;
            orc_stream_init(&st, seed, 0u, step, (uint32_t)c, ORC_PH_POP);
            uint32_t krem = is - g;
            for (uint32_t i = 0; i < is && krem > 0; ++i) {
                /* u (is - i) < krem with u = x / 2^32, exactly in 64-bit integers */
                uint32_t x = orc_stream_next(&st);
                if ((uint64_t)(is - i) * x < ((uint64_t)krem << 32)) { dead[start[c] + i] = 1; --krem; }
            }
        }
    }
    if (births > npool) { free(dead); return -1; }
    int64_t o = 0, b = 0, k = 0;
    for (int64_t c = 0; c < ncells; ++c) {
        uint32_t is = count[c], g = goal[c] > 0 ? (uint32_t)goal[c] : 0u;
        for (uint32_t j = g > is ? g - is : 0; j > 0; --j) { keys_out[o] = (uint32_t)c; ids_out[o] = pool[b++]; ++o; }
        for (uint32_t i = 0; i < is; ++i) {
            int64_t q = start[c] + i;
            if (!dead[q]) { keys_out[o] = (uint32_t)c; ids_out[o] = ids[q]; ++o; }
        }
    }
    for (int64_t q = 0; q < n; ++q) if (dead[q]) pool_out[k++] = ids[q];
    for (int64_t t = b; t < npool; ++t) pool_out[k++] = pool[t];
    (void)keys;
    *n_out = o;
    *npool_out = k;
    free(dead);
    return 0;
}
