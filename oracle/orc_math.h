/*
 * oracle/orc_math.h -- TEST INFRASTRUCTURE ONLY (the oracle).
 *
 * CPU replay of the elementary functions and samplers that the CUDA kernels of
 * this project use, written so that the same sequence of IEEE-754 single
 * precision operations runs on both sides (the oracle is compiled with
 * -ffp-contract=off; every fused multiply-add below is an explicit fmaf, which
 * is correctly rounded both in glibc and on the GPU).  This is what makes a
 * seeded GPU run replayable bit for bit on the CPU.
 *
 * The functions come from the mathematics, not from any vendor library:
 *  - log:  x = m 2^e, m in [sqrt(1/2), sqrt(2)), log m = 2 atanh(s), s=(m-1)/(m+1),
 *          atanh series truncated after s^11 (truncation < 2e-11 relative).
 *  - exp:  Cody-Waite reduction x = k ln2 + r, |r| <= ln2/2, Taylor series to r^8.
 *  - sin/cos(2 pi u): quadrant reduction on u, Taylor series on [-pi/4, pi/4].
 * The samplers:
 *  - binomial: chunked inversion (pmf recurrence from (1-q)^m, computed by binary
 *    powering); q <= 1/2 by symmetry; chunks keep (1-q)^m above 1e-26.
 *  - Poisson: counting unit-rate exponential arrivals up to lambda.
 */
#ifndef ORC_MATH_H
#define ORC_MATH_H
#include <math.h>
#include <stdint.h>
#include <string.h>
#include <limits.h>
#include "orc_rng.h"

static inline uint32_t orc_f2u(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }
static inline float orc_u2f(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }

/* uniform in (0,1]: 24 random bits, exact in float */
static inline float orc_u01_open0(uint32_t x) { return (float)((x >> 8) + 1u) * 5.9604644775390625e-08f; }
/* uniform in [0,1) */
static inline float orc_u01(uint32_t x) { return (float)(x >> 8) * 5.9604644775390625e-08f; }

#define ORC_LN2_HI 0.693145751953125f          /* ln 2 rounded to 12 significant bits: exact products with small k */
#define ORC_LN2_LO 1.4286068202862268e-06f   /* ln 2 - ORC_LN2_HI */

static inline float orc_logf(float x) {
    if (!(x > 0.0f)) return x == 0.0f ? -INFINITY : NAN;
    if (isinf(x)) return x;
    uint32_t b = orc_f2u(x);
    int e = 0;
    if ((b >> 23) == 0) {           /* subnormal: scale into the normal range */
        x = x * 16777216.0f;        /* 2^24 */
        b = orc_f2u(x);
        e = -24;
    }
    e += (int)((b >> 23) & 0xffu) - 127;
    float m = orc_u2f((b & 0x007fffffu) | 0x3f800000u); /* [1,2) */
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
    return fmaf(fe, ORC_LN2_HI, fmaf(fe, ORC_LN2_LO, lm));
}

static inline float orc_expf(float x) {
    if (x != x) return x;
    if (x > 88.5f) return INFINITY;
    if (x < -103.0f) return 0.0f;
    float kf = rintf(x * 1.4426950408889634f);     /* log2(e) */
    float r = fmaf(-kf, ORC_LN2_HI, x);
    r = fmaf(-kf, ORC_LN2_LO, r);
    /* Taylor: sum r^n / n!, n = 0..8 */
    float p = fmaf(r, 1.0f / 40320.0f, 1.0f / 5040.0f);
    p = fmaf(r, p, 1.0f / 720.0f);
    p = fmaf(r, p, 1.0f / 120.0f);
    p = fmaf(r, p, 1.0f / 24.0f);
    p = fmaf(r, p, 1.0f / 6.0f);
    p = fmaf(r, p, 0.5f);
    p = fmaf(r, p, 1.0f);
    p = fmaf(r, p, 1.0f);
    int k = (int)kf;
    /* scale by 2^k in two steps so that k down to -149 and up to 128 stay exact */
    int k1 = k / 2, k2 = k - k1;
    float s1 = orc_u2f((uint32_t)(k1 + 127) << 23);
    float s2 = orc_u2f((uint32_t)(k2 + 127) << 23);
    return (p * s1) * s2;
}

/* sin(2 pi u), cos(2 pi u) for u in [0,1) */
static inline void orc_sincos2pi(float u, float* sn, float* cs) {
    float a = u * 4.0f;
    float qf = rintf(a);
    float d = a - qf;                        /* exact, in [-1/2, 1/2] */
    float y = d * 1.5707963267948966f;   /* pi/2 */
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
    switch (q) {
        case 0: *sn = sy;  *cs = cy;  break;
        case 1: *sn = cy;  *cs = -sy; break;
        case 2: *sn = -sy; *cs = -cy; break;
        default: *sn = -cy; *cs = sy; break;
    }
}

static inline float orc_tanhf_pos(float e) {       /* e >= 0 */
    float t = orc_expf(-2.0f * e);
    return (1.0f - t) / (1.0f + t);
}
static inline float orc_tanhf(float e) { return e < 0.0f ? -orc_tanhf_pos(-e) : orc_tanhf_pos(e); }
static inline float orc_sinhf(float e) {
    float E = orc_expf(e);
    return (E - 1.0f / E) * 0.5f;
}


/* double-precision exp, same construction as orc_expf: Cody-Waite reduction with a
 * two-part ln 2 (high part with 21 trailing zero bits), Taylor series to r^13 */
#define ORC_LN2_HI_D 0.6931471803691238
#define ORC_LN2_LO_D 1.9082149292705877e-10
static inline double orc_exp_d(double x) {
    if (x != x) return x;
    if (x > 709.0) return INFINITY;
    if (x < -745.0) return 0.0;
    double kd = rint(x * 1.4426950408889634);
    double r = fma(-kd, ORC_LN2_HI_D, x);
    r = fma(-kd, ORC_LN2_LO_D, r);
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
    uint64_t b1 = (uint64_t)(k1 + 1023) << 52, b2 = (uint64_t)(k2 + 1023) << 52;
    double s1, s2;
    memcpy(&s1, &b1, 8);
    memcpy(&s2, &b2, 8);
    return (p * s1) * s2;
}

/* Per-cell stable time step of a directional drift-diffusion sweep, the reference's
 * formula (StochasticInhomogeneousDriftDiffusion.cl:124-151) evaluated in double:
 *   r = 0: h^2/(2D) (1 - 2/3);  D = 0: h/|r|;
 *   else eps = h r/(2D), temp = 1 - 1/(eps tanh eps) + 1/sinh^2 eps (<= 0 -> 1/3),
 *        dt = h/r tanh(eps) temp,
 * with tanh eps = eps - eps^3/3 and temp = 1/3 + 4 eps^2/45 for |eps| < 1e-3, where
 * the closed form cancels. */
static inline double orc_cell_timestep_d(float Df, float rf, float dxf) {
    const double D = Df, r = rf, dx = dxf;
    if (r == 0.0) return dx * dx / (2.0 * D) * (1.0 / 3.0);
    if (D == 0.0) return dx / fabs(r);
    const double eps = dx * r / (2.0 * D);
    const double a = fabs(eps);
    double th, temp;
    if (a < 1e-3) {
        th = eps - eps * eps * eps / 3.0;
        temp = 1.0 / 3.0 + 4.0 * eps * eps / 45.0;
    } else {
        const double t = orc_exp_d(-2.0 * a);
        const double tha = (1.0 - t) / (1.0 + t);
        th = eps < 0.0 ? -tha : tha;
        const double E = orc_exp_d(a);
        const double sha = (E - 1.0 / E) * 0.5;
        temp = 1.0 + (-1.0 / (th * eps) + 1.0 / (sha * sha));
        if (temp <= 0.0) temp = 1.0 / 3.0;
    }
    return dx / r * th * temp;
}
static inline float orc_cell_timestep(float D, float r, float dx) { return (float)orc_cell_timestep_d(D, r, dx); }

/* stochastic_inhomogeneous_fpe (StochasticInhomogeneousDriftDiffusion.cl:124-129):
 * StayProbability / 6 / (D / dx^2 + |r| / (2 dx)), in float */
static inline float orc_fpe_timestep(float D, float r, float dx, float stay) {
    return stay / 6.0f / (D / (dx * dx) + fabsf(r) / (2.0f * dx));
}
/* deterministic inhomogeneous solvers (:157-190): the drift formula scaled by 0.1, the
 * r == 0 formula unscaled; D == 0 with drift gives 0.1 dx / |r| (the reference divides
 * by zero there) */
static inline float orc_det_timestep(float D, float r, float dx) {
    if (r == 0.0f) return (float)orc_cell_timestep_d(D, r, dx);
    return (float)(0.1 * orc_cell_timestep_d(D, r, dx));
}

/* Binomial(n, p) by chunked inversion. */
static inline int orc_binomial(orc_stream* st, int n, float p) {
    if (n <= 0 || !(p > 0.0f)) return 0;
    if (p >= 1.0f) return n;
    int flip = p > 0.5f;
    float q = flip ? 1.0f - p : p;
    float r = q / (1.0f - q);
    float chunkf = 30.0f / q;
    int chunk = chunkf >= 2147483520.0f ? INT_MAX : (int)chunkf;
    if (chunk < 1) chunk = 1;
    int rem = n, total = 0;
    while (rem > 0) {
        int m = rem < chunk ? rem : chunk;
        float base = 1.0f - q, f = 1.0f;
        int e = m;
        while (e) {
            if (e & 1) f = f * base;
            e >>= 1;
            if (e) base = base * base;
        }
        float u = orc_u01(orc_stream_next(st));
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

/* Poisson(lambda): number of unit-rate exponential arrivals before lambda. */
static inline int orc_poisson(orc_stream* st, float lam) {
    if (!(lam > 0.0f)) return 0;
    int k = 0;
    float t = 0.0f;
    for (;;) {
        t = t - orc_logf(orc_u01_open0(orc_stream_next(st)));
        if (t > lam) break;
        k++;
        if (k == INT_MAX) break;
    }
    return k;
}

/* standard normal pair by the Box-Muller transform */
static inline void orc_normal2(orc_stream* st, float* z0, float* z1) {
    float u1 = orc_u01_open0(orc_stream_next(st));
    float u2 = orc_u01(orc_stream_next(st));
    float rad = sqrtf(-2.0f * orc_logf(u1));
    float s, c;
    orc_sincos2pi(u2, &s, &c);
    *z0 = rad * c;
    *z1 = rad * s;
}

#endif
