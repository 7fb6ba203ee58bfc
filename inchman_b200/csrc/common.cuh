// Device building blocks shared by the stochastic kernels.
//
// Random streams are Philox-4x32-10 (Salmon et al., SC'11), keyed by
// (seed, realisation) and counted by (draw, step seed, cell, phase|species|sweep),
// so every draw is a pure function of where it is used: the same results come out
// whatever the launch shape, tile size or batching (plain, wide or persistent).
//
// The elementary functions and samplers are written from the mathematics and
// evaluate a fixed sequence of IEEE single-precision operations (explicit fmaf,
// the file is compiled with -fmad=false), so a CPU replay gets the same bits:
//   log   x = m 2^e, log m = 2 atanh((m-1)/(m+1)), series to s^11
//   exp   x = k ln2 + r (two-part ln2), Taylor series to r^8
//   sin/cos(2 pi u)  quadrant reduction on u, Taylor series on [-pi/4, pi/4]
//   binomial  chunked inversion of the pmf recurrence, (1-q)^m by binary powering
//   Poisson   count of unit-rate exponential arrivals before lambda
#pragma once
#ifdef __CUDACC_RTC__
#include "gpgmp_rtc_prelude.h"    // run-time compilation: fixed-width types and limits
#else
#include <cstdint>
#include <climits>
#include <cuda_runtime.h>
#endif

namespace gpgmp {

constexpr uint32_t PH_INIT = 0x01000000u;
constexpr uint32_t PH_SSA = 0x02000000u;
constexpr uint32_t PH_DIFF = 0x03000000u;
constexpr uint32_t PH_SOURCE = 0x04000000u;
constexpr uint32_t PH_PART = 0x05000000u;
constexpr uint32_t PH_PAIR = 0x06000000u;
constexpr uint32_t PH_POP = 0x07000000u;    // population bookkeeping (individuals)

constexpr int SSA_EVENT_CAP = 1 << 22;
constexpr int SIM_EVENT_CAP = 1;
constexpr int SIM_OVERFLOW = 2;
constexpr int MAX_SPECIES = 32;
constexpr int MAX_REACTIONS = 128;

__host__ __device__ __forceinline__ void philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                                       uint32_t k0, uint32_t k1, uint32_t out[4]) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
#ifdef __CUDA_ARCH__
        uint32_t hi0 = __umulhi(0xD2511F53u, c0), lo0 = 0xD2511F53u * c0;
        uint32_t hi1 = __umulhi(0xCD9E8D57u, c2), lo1 = 0xCD9E8D57u * c2;
#else
        uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
#endif
        uint32_t n0 = hi1 ^ c1 ^ k0;
        uint32_t n2 = hi0 ^ c3 ^ k1;
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

// A stream: key fixed, counter word 0 advances, four outputs buffered.
struct Stream {
    uint32_t k0, k1, c1, c2, c3, c0;
    uint32_t buf[4];
    int idx;
    __device__ __forceinline__ void init(uint32_t key0, uint32_t key1, uint32_t ctr1, uint32_t ctr2, uint32_t ctr3) {
        k0 = key0; k1 = key1; c1 = ctr1; c2 = ctr2; c3 = ctr3; c0 = 0u; idx = 4;
    }
    __device__ __forceinline__ uint32_t next() {
        if (idx == 4) {
            philox4x32_10(c0, c1, c2, c3, k0, k1, buf);
            c0 += 1u;
            idx = 0;
        }
        uint32_t v;
        // constant-index selects keep buf in registers
        v = idx == 0 ? buf[0] : (idx == 1 ? buf[1] : (idx == 2 ? buf[2] : buf[3]));
        ++idx;
        return v;
    }
};

__device__ __forceinline__ float u01_open0(uint32_t x) { return (float)((x >> 8) + 1u) * 5.9604644775390625e-08f; }
__device__ __forceinline__ float u01(uint32_t x) { return (float)(x >> 8) * 5.9604644775390625e-08f; }

#define GPGMP_LN2_HI 0.693145751953125f
#define GPGMP_LN2_LO 1.4286068202862268e-06f

__device__ __forceinline__ float gp_logf(float x) {
    if (!(x > 0.0f)) return x == 0.0f ? -INFINITY : __int_as_float(0x7fc00000);
    if (isinf(x)) return x;
    uint32_t b = __float_as_uint(x);
    int e = 0;
    if ((b >> 23) == 0) {
        x = x * 16777216.0f;
        b = __float_as_uint(x);
        e = -24;
    }
    e += (int)((b >> 23) & 0xffu) - 127;
    float m = __uint_as_float((b & 0x007fffffu) | 0x3f800000u);
    if (m > 1.41421353816986083984375f) { m = m * 0.5f; e += 1; }
    float s = (m - 1.0f) / (m + 1.0f);
    float z = s * s;
    float p = fmaf(z, 2.0f / 11.0f, 2.0f / 9.0f);
    p = fmaf(z, p, 2.0f / 7.0f);
    p = fmaf(z, p, 2.0f / 5.0f);
    p = fmaf(z, p, 2.0f / 3.0f);
    p = fmaf(z, p, 2.0f);
    float lm = s * p;
    float fe = (float)e;
    return fmaf(fe, GPGMP_LN2_HI, fmaf(fe, GPGMP_LN2_LO, lm));
}

__device__ __forceinline__ float gp_expf(float x) {
    if (x != x) return x;
    if (x > 88.5f) return INFINITY;
    if (x < -103.0f) return 0.0f;
    float kf = rintf(x * 1.4426950408889634f);
    float r = fmaf(-kf, GPGMP_LN2_HI, x);
    r = fmaf(-kf, GPGMP_LN2_LO, r);
    float p = fmaf(r, 1.0f / 40320.0f, 1.0f / 5040.0f);
    p = fmaf(r, p, 1.0f / 720.0f);
    p = fmaf(r, p, 1.0f / 120.0f);
    p = fmaf(r, p, 1.0f / 24.0f);
    p = fmaf(r, p, 1.0f / 6.0f);
    p = fmaf(r, p, 0.5f);
    p = fmaf(r, p, 1.0f);
    p = fmaf(r, p, 1.0f);
    int k = (int)kf;
    int k1 = k / 2, k2 = k - k1;
    float s1 = __uint_as_float((uint32_t)(k1 + 127) << 23);
    float s2 = __uint_as_float((uint32_t)(k2 + 127) << 23);
    return (p * s1) * s2;
}

__device__ __forceinline__ void gp_sincos2pi(float u, float* sn, float* cs) {
    float a = u * 4.0f;
    float qf = rintf(a);
    float d = a - qf;
    float y = d * 1.5707963267948966f;
    float z = y * y;
    float ps = fmaf(z, -1.0f / 39916800.0f, 1.0f / 362880.0f);
    ps = fmaf(z, ps, -1.0f / 5040.0f);
    ps = fmaf(z, ps, 1.0f / 120.0f);
    ps = fmaf(z, ps, -1.0f / 6.0f);
    float sy = fmaf(y * z, ps, y);
    float pc = fmaf(z, 1.0f / 479001600.0f, -1.0f / 3628800.0f);
    pc = fmaf(z, pc, 1.0f / 40320.0f);
    pc = fmaf(z, pc, -1.0f / 720.0f);
    pc = fmaf(z, pc, 1.0f / 24.0f);
    pc = fmaf(z, pc, -0.5f);
    float cy = fmaf(z, pc, 1.0f);
    int q = ((int)qf) & 3;
    float s_, c_;
    if (q == 0) { s_ = sy; c_ = cy; }
    else if (q == 1) { s_ = cy; c_ = -sy; }
    else if (q == 2) { s_ = -sy; c_ = -cy; }
    else { s_ = -cy; c_ = sy; }
    *sn = s_;
    *cs = c_;
}


// double-precision exp, same construction as gp_expf (two-part ln 2 with 21 trailing
// zero bits in the high part, Taylor series to r^13)
__device__ __forceinline__ double gp_exp_d(double x) {
    if (x != x) return x;
    if (x > 709.0) return INFINITY;
    if (x < -745.0) return 0.0;
    double kd = rint(x * 1.4426950408889634);
    double r = fma(-kd, 0.6931471803691238, x);
    r = fma(-kd, 1.9082149292705877e-10, r);
    double p = fma(r, 1.0 / 6227020800.0, 1.0 / 479001600.0);
    p = fma(r, p, 1.0 / 39916800.0);
    p = fma(r, p, 1.0 / 3628800.0);
    p = fma(r, p, 1.0 / 362880.0);
    p = fma(r, p, 1.0 / 40320.0);
    p = fma(r, p, 1.0 / 5040.0);
    p = fma(r, p, 1.0 / 720.0);
    p = fma(r, p, 1.0 / 120.0);
    p = fma(r, p, 1.0 / 24.0);
    p = fma(r, p, 1.0 / 6.0);
    p = fma(r, p, 0.5);
    p = fma(r, p, 1.0);
    p = fma(r, p, 1.0);
    int k = (int)kd;
    int k1 = k / 2, k2 = k - k1;
    double s1 = __longlong_as_double((long long)(k1 + 1023) << 52);
    double s2 = __longlong_as_double((long long)(k2 + 1023) << 52);
    return (p * s1) * s2;
}

__device__ __forceinline__ float gp_tanhf(float e) {
    float a = e < 0.0f ? -e : e;
    float t = gp_expf(-2.0f * a);
    float v = (1.0f - t) / (1.0f + t);
    return e < 0.0f ? -v : v;
}
__device__ __forceinline__ float gp_sinhf(float e) {
    float E = gp_expf(e);
    return (E - 1.0f / E) * 0.5f;
}

__device__ __forceinline__ int binomial(Stream& st, int n, float p) {
    if (n <= 0 || !(p > 0.0f)) return 0;
    if (p >= 1.0f) return n;
    const bool flip = p > 0.5f;
    const float q = flip ? 1.0f - p : p;
    const float r = q / (1.0f - q);
    const float chunkf = 30.0f / q;
    int chunk = chunkf >= 2147483520.0f ? INT_MAX : (int)chunkf;
    if (chunk < 1) chunk = 1;
    int rem = n, total = 0;
    while (rem > 0) {
        const int m = rem < chunk ? rem : chunk;
        float base = 1.0f - q, f = 1.0f;
        int e = m;
        while (e) {
            if (e & 1) f = f * base;
            e >>= 1;
            if (e) base = base * base;
        }
        const float u = u01(st.next());
        int k = 0;
        float cdf = f;
        while (u >= cdf && k < m) {
            f = f * ((float)(m - k) * r) / (float)(k + 1);
            k++;
            cdf = cdf + f;
        }
        total += k;
        rem -= m;
    }
    return flip ? n - total : total;
}

__device__ __forceinline__ int poisson(Stream& st, float lam) {
    if (!(lam > 0.0f)) return 0;
    int k = 0;
    float t = 0.0f;
    for (;;) {
        t = t - gp_logf(u01_open0(st.next()));
        if (t > lam) break;
        k++;
        if (k == INT_MAX) break;
    }
    return k;
}

__device__ __forceinline__ void normal2(Stream& st, float* z0, float* z1) {
    float u1 = u01_open0(st.next());
    float u2 = u01(st.next());
    float rad = sqrtf(-2.0f * gp_logf(u1));
    float s, c;
    gp_sincos2pi(u2, &s, &c);
    *z0 = rad * c;
    *z1 = rad * s;
}

}  // namespace gpgmp
