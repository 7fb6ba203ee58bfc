/*
 * oracle/orc_det.c -- TEST INFRASTRUCTURE ONLY (the oracle).
 *
 * Deterministic reaction-diffusion oracles:
 *  - Gray-Scott, forward Euler, 5-point periodic Laplacian (h = 1), in float (in
 *    the GPU kernels' operation order, bit-exact) and double, and the double-precision discrete adjoint of the loss
 *    L = sum (u_N - u*)^2 + (v_N - v*)^2 with respect to (F, k, Du, Dv, vx, vy), with
 *    checkpoints every `checkpoint_every` steps and per-segment recomputation.
 *    The network is the reference's Gray-Scott model (exec/src/tests/
 *    GrayScottModel.cpp:14-60: U+2V->3V, U->0 at F, V->0 at F+k, 0->U at F),
 *    whose deterministic laws (Reaction.cpp:145-162) give the ODE right-hand side
 *    -u v^2 + F (1 - u), u v^2 - (F + k) v; a constant drift (vx, vy) enters by
 *    central differences (Deterministic.cl:71-136 with constant velocity).
 *  - The reference's deterministic event loops (DiffusionModel.cpp:1414-1603):
 *    homogeneous (HomogeneousSolver.cpp:168-192 common time step,
 *    Deterministic.cl:17-65 stencil, one diffusion per event unless flags bit 3 asks
 *    for the reference's repetition of the all-species stencil once per due
 *    species) and inhomogeneous (InhomogeneousSolver.cpp:254-427 X/Y clocks,
 *    StochasticInhomogeneousDriftDiffusion.cl:157-190 time steps, Deterministic.cl:
 *    71-136 drift-diffusion sweeps, written out of place), with RK4
 *    (Deterministic.cl:143-238) or alpha-QSS (:240-522) reaction windows.  The
 *    reference runs no reactions in its inhomogeneous deterministic solvers
 *    (Solver.cpp:250-266); flags bit 5 restores that.
 *  The sweep and alpha-QSS restatements use float arithmetic in the order the CUDA
 *  kernels use; the RK4 restatement keeps the reference's double-literal evaluation.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "gpgmp_oracle.h"

#define IDX(x, y, N) ((size_t)(((y) + (N)) % (N)) * (N) + (size_t)(((x) + (N)) % (N)))

/* The float32 forward as the GPU's packed-FP32x2 kernels compute it (gs_update2f in
 * inchman_b200/csrc/gs_f32x2.cuh, used by the register-resident, column-walk and batched
 * float32 kernels): the same float operations in the same order, each fused
 * multiply-add an fmaf, so the two agree bit for bit.  Per cell, with L/R the x-1/x+1
 * and U/D the y-1/y+1 neighbours (periodic):
 *   lu = fma(-4, u, (uL + uR) + (uU + uD)),  uvv = u * (v * v)
 *   a  = fma(dt Du, lu, fma(-(dt F), u, dt F)),  b = fma(-(dt (F + k)), v, (dt Dv) * lv)
 *   drift: a = fma(hx, uL - uR, fma(hy, uU - uD, a)) (b likewise), hx = (dt vx) 0.5
 *   u' = u + fma(-dt, uvv, a),  v' = v + fma(dt, uvv, b)
 * This is the explicit Euler step of Deterministic.cl:17-65 plus the Gray-Scott
 * right-hand side of GrayScottModel.cpp:14-60 (Reaction.cpp:145-162 laws). */
static inline void gs_cell_f32x(float du, float dv, float hx, float hy, float dt, float mdt, float dtF, float mdtF,
                                float mdtFk, int drift, float uL, float uR, float uU, float uC, float uD, float vL,
                                float vR, float vU, float vC, float vD, float* un, float* vn) {
    const float uvv = uC * (vC * vC);
    const float lu = fmaf(-4.0f, uC, (uL + uR) + (uU + uD));
    const float lv = fmaf(-4.0f, vC, (vL + vR) + (vU + vD));
    float a = fmaf(du, lu, fmaf(mdtF, uC, dtF));
    float b = fmaf(mdtFk, vC, dv * lv);
    if (drift) {
        a = fmaf(hx, uL - uR, fmaf(hy, uU - uD, a));
        b = fmaf(hx, vL - vR, fmaf(hy, vU - vD, b));
    }
    *un = uC + fmaf(mdt, uvv, a);
    *vn = vC + fmaf(dt, uvv, b);
}

/* One row y of the step; the interior columns have no wrap-around, so the compiler
 * vectorises them (the fma clone uses the CPU's fused multiply-add instructions). */
__attribute__((target_clones("fma", "default")))
static void gs_row_f32x(int N, int y, float du, float dv, float hx, float hy, float dt, float mdt, float dtF,
                        float mdtF, float mdtFk, int drift, const float* restrict u, const float* restrict v,
                        float* restrict u2, float* restrict v2) {
    const float* restrict uc = u + (size_t)y * N;
    const float* restrict vc = v + (size_t)y * N;
    const float* restrict uu = u + (size_t)((y + N - 1) % N) * N;
    const float* restrict vu = v + (size_t)((y + N - 1) % N) * N;
    const float* restrict ud = u + (size_t)((y + 1) % N) * N;
    const float* restrict vd = v + (size_t)((y + 1) % N) * N;
    float* restrict uo = u2 + (size_t)y * N;
    float* restrict vo = v2 + (size_t)y * N;
    if (drift) {
        for (int x = 1; x < N - 1; ++x)
            gs_cell_f32x(du, dv, hx, hy, dt, mdt, dtF, mdtF, mdtFk, 1, uc[x - 1], uc[x + 1], uu[x], uc[x], ud[x],
                         vc[x - 1], vc[x + 1], vu[x], vc[x], vd[x], &uo[x], &vo[x]);
    } else {
        for (int x = 1; x < N - 1; ++x)
            gs_cell_f32x(du, dv, hx, hy, dt, mdt, dtF, mdtF, mdtFk, 0, uc[x - 1], uc[x + 1], uu[x], uc[x], ud[x],
                         vc[x - 1], vc[x + 1], vu[x], vc[x], vd[x], &uo[x], &vo[x]);
    }
    const int edge[2] = {0, N - 1};
    for (int e = 0; e < (N > 1 ? 2 : 1); ++e) {
        const int x = edge[e], xl = (x + N - 1) % N, xr = (x + 1) % N;
        gs_cell_f32x(du, dv, hx, hy, dt, mdt, dtF, mdtF, mdtFk, drift, uc[xl], uc[xr], uu[x], uc[x], ud[x], vc[xl],
                     vc[xr], vu[x], vc[x], vd[x], &uo[x], &vo[x]);
    }
}

void orc_gs_forward_f32(int N, int steps, float F, float k, float Du, float Dv, float vx, float vy, float dt,
                         float* u, float* v) {
    const size_t n = (size_t)N * N;
    /* coefficients as the kernels form them from the float parameters (GSCoef2) */
    const float du = dt * Du, dv = dt * Dv, hx = dt * vx * 0.5f, hy = dt * vy * 0.5f;
    const float mdt = -dt, dtF = dt * F, mdtF = -(dt * F), mdtFk = -(dt * (F + k));
    const int drift = vx != 0.0f || vy != 0.0f;
    float* buf = (float*)malloc(sizeof(float) * 2 * n);
    float *cu = u, *cv = v, *nu = buf, *nv = buf + n;
    /* one parallel region for the whole solve: each thread keeps the same rows every
     * step, and the barrier at the end of the loop over rows separates the steps */
    #pragma omp parallel firstprivate(cu, cv, nu, nv)
    for (int s = 0; s < steps; ++s) {
        #pragma omp for schedule(static)
        for (int y = 0; y < N; ++y)
            gs_row_f32x(N, y, du, dv, hx, hy, dt, mdt, dtF, mdtF, mdtFk, drift, cu, cv, nu, nv);
        float* t = cu; cu = nu; nu = t;
        t = cv; cv = nv; nv = t;
    }
    if (steps % 2 == 1) {    /* the result is in the work buffer */
        cu = buf;
        cv = buf + n;
    }
    if (cu != u) {
        memcpy(u, cu, sizeof(float) * n);
        memcpy(v, cv, sizeof(float) * n);
    }
    free(buf);
}

static void gs_step_f64(int N, double F, double k, double Du, double Dv, double vx, double vy, double dt,
                        const double* u, const double* v, double* u2, double* v2) {
    #pragma omp parallel for schedule(static)
    for (int y = 0; y < N; ++y)
        for (int x = 0; x < N; ++x) {
            size_t i = (size_t)y * N + x;
            double uc = u[i], vc = v[i];
            double lu = u[IDX(x - 1, y, N)] + u[IDX(x + 1, y, N)] + u[IDX(x, y - 1, N)] + u[IDX(x, y + 1, N)] - 4.0 * uc;
            double lv = v[IDX(x - 1, y, N)] + v[IDX(x + 1, y, N)] + v[IDX(x, y - 1, N)] + v[IDX(x, y + 1, N)] - 4.0 * vc;
            double uvv = uc * vc * vc;
            double au = vx * (u[IDX(x + 1, y, N)] - u[IDX(x - 1, y, N)]) * 0.5 + vy * (u[IDX(x, y + 1, N)] - u[IDX(x, y - 1, N)]) * 0.5;
            double av = vx * (v[IDX(x + 1, y, N)] - v[IDX(x - 1, y, N)]) * 0.5 + vy * (v[IDX(x, y + 1, N)] - v[IDX(x, y - 1, N)]) * 0.5;
            u2[i] = uc + dt * (Du * lu - au - uvv + F * (1.0 - uc));
            v2[i] = vc + dt * (Dv * lv - av + uvv - (F + k) * vc);
        }
}

void orc_gs_forward_f64(int N, int steps, double F, double k, double Du, double Dv, double vx, double vy, double dt,
                        double* u, double* v) {
    const size_t n = (size_t)N * N;
    double* u2 = (double*)malloc(sizeof(double) * n);
    double* v2 = (double*)malloc(sizeof(double) * n);
    for (int s = 0; s < steps; ++s) {
        gs_step_f64(N, F, k, Du, Dv, vx, vy, dt, u, v, u2, v2);
        memcpy(u, u2, sizeof(double) * n);
        memcpy(v, v2, sizeof(double) * n);
    }
    free(u2); free(v2);
}

double orc_gs_loss_grad_f64(int N, int steps, double F, double k, double Du, double Dv, double vx, double vy,
                            double dt, const double* u0, const double* v0, const double* ut, const double* vt,
                            int ck, double* grad6) {
    const size_t n = (size_t)N * N;
    if (ck <= 0) ck = steps;
    const int nseg = (steps + ck - 1) / ck;
    double* cu = (double*)malloc(sizeof(double) * n * (size_t)nseg);
    double* cv = (double*)malloc(sizeof(double) * n * (size_t)nseg);
    double* su = (double*)malloc(sizeof(double) * n * (size_t)(ck + 1));
    double* sv = (double*)malloc(sizeof(double) * n * (size_t)(ck + 1));
    double* lu = (double*)malloc(sizeof(double) * n);
    double* lv = (double*)malloc(sizeof(double) * n);
    double* lu2 = (double*)malloc(sizeof(double) * n);
    double* lv2 = (double*)malloc(sizeof(double) * n);
    /* forward with checkpoints at steps 0, ck, 2ck, ... */
    memcpy(su, u0, sizeof(double) * n);
    memcpy(sv, v0, sizeof(double) * n);
    for (int s = 0; s < steps; ++s) {
        if (s % ck == 0) {
            memcpy(cu + (size_t)(s / ck) * n, su, sizeof(double) * n);
            memcpy(cv + (size_t)(s / ck) * n, sv, sizeof(double) * n);
        }
        gs_step_f64(N, F, k, Du, Dv, vx, vy, dt, su, sv, su + n, sv + n);
        memcpy(su, su + n, sizeof(double) * n);
        memcpy(sv, sv + n, sizeof(double) * n);
    }
    double loss = 0.0;
    for (size_t i = 0; i < n; ++i) {
        double du = su[i] - ut[i], dv = sv[i] - vt[i];
        loss += du * du + dv * dv;
        lu[i] = 2.0 * du;
        lv[i] = 2.0 * dv;
    }
    double gF = 0, gk = 0, gDu = 0, gDv = 0, gvx = 0, gvy = 0;
    for (int seg = nseg - 1; seg >= 0; --seg) {
        int s0 = seg * ck, s1 = s0 + ck < steps ? s0 + ck : steps;
        int len = s1 - s0;
        memcpy(su, cu + (size_t)seg * n, sizeof(double) * n);
        memcpy(sv, cv + (size_t)seg * n, sizeof(double) * n);
        for (int j = 0; j < len - 1; ++j)
            gs_step_f64(N, F, k, Du, Dv, vx, vy, dt, su + (size_t)j * n, sv + (size_t)j * n,
                        su + (size_t)(j + 1) * n, sv + (size_t)(j + 1) * n);
        for (int j = len - 1; j >= 0; --j) {
            const double* u = su + (size_t)j * n;
            const double* v = sv + (size_t)j * n;
            double aF = 0, ak = 0, aDu = 0, aDv = 0, avx = 0, avy = 0;
            #pragma omp parallel for schedule(static) reduction(+:aF, ak, aDu, aDv, avx, avy)
            for (int y = 0; y < N; ++y)
                for (int x = 0; x < N; ++x) {
                    size_t i = (size_t)y * N + x;
                    double uc = u[i], vc = v[i];
                    double lapu = u[IDX(x - 1, y, N)] + u[IDX(x + 1, y, N)] + u[IDX(x, y - 1, N)] + u[IDX(x, y + 1, N)] - 4.0 * uc;
                    double lapv = v[IDX(x - 1, y, N)] + v[IDX(x + 1, y, N)] + v[IDX(x, y - 1, N)] + v[IDX(x, y + 1, N)] - 4.0 * vc;
                    double a = lu[i], b = lv[i];
                    double lapa = lu[IDX(x - 1, y, N)] + lu[IDX(x + 1, y, N)] + lu[IDX(x, y - 1, N)] + lu[IDX(x, y + 1, N)] - 4.0 * a;
                    double lapb = lv[IDX(x - 1, y, N)] + lv[IDX(x + 1, y, N)] + lv[IDX(x, y - 1, N)] + lv[IDX(x, y + 1, N)] - 4.0 * b;
                    double dxa = (lu[IDX(x + 1, y, N)] - lu[IDX(x - 1, y, N)]) * 0.5;
                    double dya = (lu[IDX(x, y + 1, N)] - lu[IDX(x, y - 1, N)]) * 0.5;
                    double dxb = (lv[IDX(x + 1, y, N)] - lv[IDX(x - 1, y, N)]) * 0.5;
                    double dyb = (lv[IDX(x, y + 1, N)] - lv[IDX(x, y - 1, N)]) * 0.5;
                    double dxu = (u[IDX(x + 1, y, N)] - u[IDX(x - 1, y, N)]) * 0.5;
                    double dyu = (u[IDX(x, y + 1, N)] - u[IDX(x, y - 1, N)]) * 0.5;
                    double dxv = (v[IDX(x + 1, y, N)] - v[IDX(x - 1, y, N)]) * 0.5;
                    double dyv = (v[IDX(x, y + 1, N)] - v[IDX(x, y - 1, N)]) * 0.5;
                    lu2[i] = a + dt * (Du * lapa + vx * dxa + vy * dya + a * (-vc * vc - F) + b * (vc * vc));
                    lv2[i] = b + dt * (Dv * lapb + vx * dxb + vy * dyb + a * (-2.0 * uc * vc) + b * (2.0 * uc * vc - (F + k)));
                    aF += dt * (a * (1.0 - uc) - b * vc);
                    ak += dt * (-b * vc);
                    aDu += dt * a * lapu;
                    aDv += dt * b * lapv;
                    avx += dt * (-a * dxu - b * dxv);
                    avy += dt * (-a * dyu - b * dyv);
                }
            gF += aF; gk += ak; gDu += aDu; gDv += aDv; gvx += avx; gvy += avy;
            double* t;
            t = lu; lu = lu2; lu2 = t;
            t = lv; lv = lv2; lv2 = t;
        }
    }
    grad6[0] = gF; grad6[1] = gk; grad6[2] = gDu; grad6[3] = gDv; grad6[4] = gvx; grad6[5] = gvy;
    free(cu); free(cv); free(su); free(sv); free(lu); free(lv); free(lu2); free(lv2);
    return loss;
}

/* Deterministic.cl:71-136 for one species and direction, out of place, mirror
 * neighbours: s' = s + dt (D_l s_l + D_r s_r - 2 D s) / dx^2 - dt (r_r s_r - r_l s_l) / (2 dx). */
void orc_det_sweep(const orc_model* m, const float* in, float* out, int species, int sweep_y, float dt, float dx,
                   const float* D, const float* rv) {
    const int W = m->width, H = m->height, S = m->num_species;
    const size_t area = (size_t)W * H;
    memcpy(out, in, sizeof(float) * area * S);
    const float* p = in + (size_t)species * area;
    float* o = out + (size_t)species * area;
    const float* Dp = D + (size_t)species * area;
    const float* rp = rv + (size_t)species * area;
    const float dx2 = dx * dx;
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            const int c = x + y * W;
            int lo, hi;
            if (!sweep_y) { lo = x > 0 ? c - 1 : c + 1; hi = x < W - 1 ? c + 1 : c - 1; }
            else { lo = y > 0 ? c - W : c + W; hi = y < H - 1 ? c + W : c - W; }
            const float sl = p[lo] * Dp[lo], sr = p[hi] * Dp[hi], sh = p[c] * Dp[c];
            const float lap = sl + sr - 2.0f * sh;
            const float drift = rp[hi] * p[hi] - rp[lo] * p[lo];
            o[c] = p[c] + dt * lap / dx2 - dt * drift / (2.0f * dx);
        }
}

/* alpha-QSS (Mott & Oran 2001) as Deterministic.cl:240-522 runs it per cell: the
 * production/destruction split of Solver.cpp:961-1004 with the laws of
 * Reaction.cpp:145-162.  A retried step restarts its predictor from the saved start
 * state with the reduced step size (Mott & Oran).  literal = 1 keeps the reference's
 * predictor (current q, d and the outer step's size, :381-387) and its corrector
 * coefficient as printed (`180.*+rtaub`, :424).  Returns 1 if the step control did
 * not finish within ORC_AQSS_MAX_ITER corrector passes. */
#define ORC_AQSS_MAX_ITER 100000
static void orc_aqss_rhs(const orc_model* m, const uint32_t* on, const float* y, float* q, float* d) {
    const int S = m->num_species;
    for (int i = 0; i < S; ++i) { q[i] = 0.0f; d[i] = 0.0f; }
    for (int k = 0; k < m->num_reactions; ++k) {
        if (!orc_reaction_on(on, k)) continue;     /* localised reaction, off in this cell */
        const orc_reaction* rc = &m->reactions[k];
        float law = rc->rate;
        for (int j = 0; j < rc->num_reactants; ++j)
            for (int a = 0; a < rc->reactant_stoich[j]; ++a) law *= y[rc->reactant_species[j]];
        for (int pass = 0; pass < 2; ++pass) {
            const int cnt = pass == 0 ? rc->num_reactants : rc->num_products;
            for (int j = 0; j < cnt; ++j) {
                const int sp = pass == 0 ? rc->reactant_species[j] : rc->product_species[j];
                int seen = 0;
                for (int a = 0; a < rc->num_reactants && !seen; ++a)
                    if (rc->reactant_species[a] == sp && (pass == 1 || a < j)) seen = 1;
                for (int a = 0; a < rc->num_products && !seen && pass == 1; ++a)
                    if (rc->product_species[a] == sp && a < j) seen = 1;
                if (seen) continue;
                int net = 0;
                for (int a = 0; a < rc->num_products; ++a) if (rc->product_species[a] == sp) net += rc->product_stoich[a];
                for (int a = 0; a < rc->num_reactants; ++a) if (rc->reactant_species[a] == sp) net -= rc->reactant_stoich[a];
                if (net > 0) q[sp] += (float)net * law;
                else if (net < 0) d[sp] += (float)(-net) * law;
            }
        }
    }
}
static float orc_aqss_alpha(float r) {
    return (180.0f + r * (60.0f + r * (11.0f + r))) / (360.0f + r * (60.0f + r * (12.0f + r)));
}
static int orc_aqss_cell_on(const orc_model* m, const uint32_t* on, float* y, float dtg, int literal) {
    const int S = m->num_species;
    const float epsmin = 1e-2f, sqreps = 0.5f, epscl = 100.0f, epsmax = 10.0f, tfd = 1.000008f, dtmin = 1e-15f,
                ymin = 1e-20f;
    const int itermax = 2;
    float q[64], d[64], ys[64], qs[64], ds[64], rtaus[64], scr[64], y1[64];
    float tn = 0.0f;
    for (int i = 0; i < S; ++i) y[i] = fmaxf(y[i], ymin);
    orc_aqss_rhs(m, on, y, q, d);
    float scrtch = 1e-25f;
    for (int i = 0; i < S; ++i) {
        const float ascr = fabsf(q[i]);
        const float scr2 = copysignf(1.0f / y[i], 0.1f * epsmin * ascr - d[i]);
        const float scr1 = scr2 * d[i];
        scrtch = fmaxf(fmaxf(scr1, -fabsf(ascr - d[i]) * scr2), scrtch);
    }
    float dt = fminf(sqreps / scrtch, dtg);
    int passes = 0;
    while (dtg > tn * tfd) {
        const float ts = tn, dtcurrent = dt;
        for (int i = 0; i < S; ++i) { ys[i] = y[i]; qs[i] = q[i]; ds[i] = d[i]; rtaus[i] = dtcurrent * d[i] / y[i]; }
        while (dtg > tn * tfd) {
            if (++passes > ORC_AQSS_MAX_ITER) return 1;
            for (int i = 0; i < S; ++i) {
                if (literal) {
                    const float rtaui = dtcurrent * d[i] / y[i];
                    scr[i] = (q[i] - d[i]) / (1.0f + orc_aqss_alpha(rtaui) * rtaui);
                } else {
                    const float rtaui = dt * ds[i] / ys[i];
                    scr[i] = (qs[i] - ds[i]) / (1.0f + orc_aqss_alpha(rtaui) * rtaui);
                }
            }
            float eps = 1e-10f;
            for (int it = 0; it < itermax; ++it) {
                for (int i = 0; i < S; ++i) y[i] = fmaxf(ys[i] + dt * scr[i], ymin);
                if (it == 0) { tn = ts + dt; for (int i = 0; i < S; ++i) y1[i] = y[i]; }
                orc_aqss_rhs(m, on, y, q, d);
                eps = 1e-10f;
                for (int i = 0; i < S; ++i) {
                    const float rtaub = 0.5f * (rtaus[i] + dt * d[i] / y[i]);
                    const float alpha = literal ? (180.0f * rtaub * (60.0f + rtaub * (11.0f + rtaub))) /
                                                      (360.0f + rtaub * (60.0f + rtaub * (12.0f + rtaub)))
                                                : orc_aqss_alpha(rtaub);
                    const float qt = qs[i] * (1.0f - alpha) + q[i] * alpha;
                    const float pb = rtaub / dt;
                    scr[i] = (qt - ys[i] * pb) / (1.0f + alpha * rtaub);
                }
            }
            for (int i = 0; i < S; ++i) {
                const float scr2 = fmaxf(ys[i] + dt * scr[i], 0.0f);
                float scr1 = fabsf(scr2 - y1[i]);
                y[i] = fmaxf(scr2, ymin);
                if (0.25f * (ys[i] + y[i]) > ymin) {
                    scr1 = scr1 / y[i];
                    eps = fmaxf(0.5f * (scr1 + fminf(fabsf(q[i] - d[i]) / (q[i] + d[i] + 1e-30f), scr1)), eps);
                }
            }
            eps = eps * epscl;
            if (dt <= dtmin + 1e-16f * tn) { dt = dtg - ts; dt = fminf(dtmin, fabsf(dt)); }
            const float stab = 0.01f;
            if (eps <= epsmax && stab <= 1.0f) {
                if (dtg <= tn * tfd) break;
            } else {
                tn = ts;
            }
            const float rteps = sqrtf(eps);
            float dto = dt;
            dt = fminf(fminf(dt * (1.0f / rteps + 0.005f), tfd * (dtg - tn)), dto / (stab + 0.001f));
            if (eps <= epsmax && stab <= 1.0f) break;
            dto = dt / dto;
            for (int i = 0; i < S; ++i) rtaus[i] *= dto;
        }
        orc_aqss_rhs(m, on, y, q, d);
    }
    return 0;
}
int orc_aqss_cell(const orc_model* m, float* y, float dtg, int literal) {
    return orc_aqss_cell_on(m, NULL, y, dtg, literal);
}
/* one alpha-QSS window for every cell of one realisation's state [S][area] */
int orc_aqss(const orc_model* m, float* state, float dtg, int literal) {
    const int S = m->num_species;
    const size_t area = (size_t)m->width * m->height;
    int bad = 0;
    if (m->num_reactions <= 0) return 0;
    #pragma omp parallel for schedule(dynamic, 64) reduction(|:bad)
    for (int64_t c = 0; c < (int64_t)area; ++c) {
        float y[64];
        uint32_t on[4];
        orc_cell_reactions(m, (size_t)c, on);
        for (int i = 0; i < S; ++i) y[i] = state[c + (size_t)i * area];
        bad |= orc_aqss_cell_on(m, on, y, dtg, literal);
        for (int i = 0; i < S; ++i) state[c + (size_t)i * area] = y[i];
    }
    return bad;
}

/* InhomogeneousSolver with a deterministic type: fields and first time steps as
 * InhomogeneousSolver.cpp:164-212, X/Y sweeps when due (:254-427, no seed), reaction
 * windows by RK4 (type 5) or alpha-QSS (type 6) unless flags bit 5. */
static int orc_det_inhom_solve(const orc_model* m, float* state, float* snaps, float* snap_times, int max_snaps,
                               int* nsnap, int64_t* steps_out) {
    const int S = m->num_species;
    const size_t area = (size_t)m->width * m->height;
    const int aqss = m->solver_type == 6, react = !(m->flags & 32);
    float *Fdx = (float*)malloc(sizeof(float) * S * area), *Fdy = (float*)malloc(sizeof(float) * S * area);
    float *Frx = (float*)malloc(sizeof(float) * S * area), *Fry = (float*)malloc(sizeof(float) * S * area);
    float *nx = (float*)calloc(S, sizeof(float)), *ny = (float*)calloc(S, sizeof(float));
    float *sdx = (float*)calloc(S, sizeof(float)), *sdy = (float*)calloc(S, sizeof(float));
    float *ddx = (float*)calloc(S, sizeof(float)), *ddy = (float*)calloc(S, sizeof(float));
    float* next = (float*)calloc(S, sizeof(float));
    float* tmp = (float*)malloc(sizeof(float) * S * area);
    for (int i = 0; i < S; ++i) {
        orc_rep_diffusivity_drift(m, i, Fdx, Fdy, Frx, Fry);
        sdx[i] = orc_rep_timestep(m, i, 0, Fdx, Frx);
        sdy[i] = orc_rep_timestep(m, i, 1, Fdy, Fry);
        ddx[i] = sdx[i]; ddy[i] = sdy[i];
        nx[i] = sdx[i]; ny[i] = sdy[i];
        next[i] = nx[i] < ny[i] ? nx[i] : ny[i];
    }
    const float dxw = m->physical_length / (float)m->width, dyw = m->physical_length / (float)m->height;
    int ns = 0, bad = 0;
#define SNAP(t) do { if (ns < max_snaps) { memcpy(snaps + (size_t)ns * S * area, state, sizeof(float) * S * area); \
                      snap_times[ns] = (t); } ns++; } while (0)
    SNAP(0.f);
    float simTime = 0.f, outputLast = 0.f;
    int64_t n = 0;
    while ((m->max_steps < 0 || n < m->max_steps) && simTime < m->max_time) {
        n++;
        float mindt = next[0];
        int minspec = 0;
        for (int i = 1; i < S; ++i) if (next[i] < mindt) { mindt = next[i]; minspec = i; }
        int ev = 0;
        float mo = outputLast + m->output_interval;
        if (mo < mindt) { mindt = mo; ev = 1; }
        float deltat = mindt - simTime;
        if (m->num_reactions > 0 && react) {
            if (aqss) bad |= orc_aqss(m, state, deltat, (m->flags & 16) != 0);
            else orc_ref_rk4(m, state, deltat);
        }
        if (ev == 0) {
            for (int i = 0; i < S; ++i) {
                if (!(i == minspec || next[i] <= mindt)) continue;
                if (!(next[i] > 0)) continue;
                if (nx[i] <= mindt) {
                    orc_det_sweep(m, state, tmp, i, 0, ddx[i], dxw, Fdx, Frx);
                    memcpy(state, tmp, sizeof(float) * S * area);
                    nx[i] += sdx[i];
                    ddx[i] = sdx[i];
                }
                if (ny[i] <= mindt) {
                    orc_det_sweep(m, state, tmp, i, 1, ddy[i], dyw, Fdy, Fry);
                    memcpy(state, tmp, sizeof(float) * S * area);
                    ny[i] += sdy[i];
                    ddy[i] = sdy[i];
                }
                next[i] = nx[i] < ny[i] ? nx[i] : ny[i];
            }
        } else if (simTime >= outputLast + m->output_interval) {
            SNAP(mindt);
            outputLast += m->output_interval;
        }
        simTime = mindt;
        if ((m->flags & 4) && bad) break;
    }
    SNAP(simTime);
#undef SNAP
    *nsnap = ns;
    *steps_out = n;
    free(Fdx); free(Fdy); free(Frx); free(Fry); free(nx); free(ny); free(sdx); free(sdy); free(ddx); free(ddy);
    free(next); free(tmp);
    return bad;
}

int orc_det_solve(const orc_model* m, float* state, float* snaps, float* snap_times, int max_snaps,
                  int* nsnap, int64_t* steps_out) {
    const int ty = m->solver_type;
    if (ty == 5 || ty == 6) return orc_det_inhom_solve(m, state, snaps, snap_times, max_snaps, nsnap, steps_out);
    const int aqss = ty == 4;
    const int S = m->num_species;
    const size_t area = (size_t)m->width * m->height;
    const float h = m->physical_length / (float)m->width;
    float dtd = 0.f;
    for (int i = 0; i < S; ++i) {
        float d = m->diffusion[i] > 0 ? (float)1e-2f * h * h / (4.f * m->diffusion[i]) : m->max_time;
        if (i == 0 || d < dtd) dtd = d;
    }
    float* next = (float*)malloc(sizeof(float) * S);
    for (int i = 0; i < S; ++i) next[i] = dtd;
    float* tmp = (float*)malloc(sizeof(float) * S * area);
    int ns = 0;
#define SNAP(t) do { if (ns < max_snaps) { memcpy(snaps + (size_t)ns * S * area, state, sizeof(float) * S * area); \
                      snap_times[ns] = (t); } ns++; } while (0)
    SNAP(0.f);
    float simTime = 0.f, outputLast = 0.f;
    int64_t n = 0;
    while ((m->max_steps < 0 || n < m->max_steps) && simTime < m->max_time) {
        n++;
        float mindt = next[0];
        int minspec = 0;
        for (int i = 1; i < S; ++i) if (next[i] < mindt) { mindt = next[i]; minspec = i; }
        int ev = 0;
        float mo = outputLast + m->output_interval;
        if (mo < mindt) { mindt = mo; ev = 1; }
        float deltat = mindt - simTime;
        if (m->num_reactions > 0) {
            if (aqss) orc_aqss(m, state, deltat, (m->flags & 16) != 0);
            else orc_ref_rk4(m, state, deltat);
        }
        if (ev == 0) {
            int applied = 0;
            for (int i = 0; i < S; ++i) {
                if (!(i == minspec || next[i] <= mindt)) continue;
                if (!(next[i] > 0)) continue;
                if (!applied || (m->flags & 8)) {
                    orc_ref_det_diffuse(m, state, tmp, dtd, 0);
                    memcpy(state, tmp, sizeof(float) * S * area);
                    applied = 1;
                }
                next[i] += dtd;
            }
        } else if (simTime >= outputLast + m->output_interval) {
            SNAP(mindt);
            outputLast += m->output_interval;
        }
        simTime = mindt;
    }
    SNAP(simTime);
#undef SNAP
    *nsnap = ns;
    *steps_out = n;
    free(next); free(tmp);
    return 0;
}
