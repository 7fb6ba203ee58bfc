/*
 * oracle/orc_det.c -- TEST INFRASTRUCTURE ONLY (the oracle).
 *
 * Deterministic reaction-diffusion oracles:
 *  - Gray-Scott, forward Euler, 5-point periodic Laplacian (h = 1), in float and
 *    double, and the double-precision discrete adjoint of the loss
 *    L = sum (u_N - u*)^2 + (v_N - v*)^2 with respect to (F, k, Du, Dv, vx, vy), with
 *    checkpoints every `checkpoint_every` steps and per-segment recomputation.
 *    The network is the reference's Gray-Scott model (exec/src/tests/
 *    GrayScottModel.cpp:14-60: U+2V->3V, U->0 at F, V->0 at F+k, 0->U at F),
 *    whose deterministic laws (Reaction.cpp:145-162) give the ODE right-hand side
 *    -u v^2 + F (1 - u), u v^2 - (F + k) v; a constant drift (vx, vy) enters by
 *    central differences (Deterministic.cl:71-136 with constant velocity).
 *  - The reference's deterministic RK4 event loop (DiffusionModel.cpp:1414-1603,
 *    HomogeneousSolver.cpp:168-192 common time step, Deterministic.cl:17-65 and
 *    :179-238), with one diffusion per event unless flags bit 3 asks for the
 *    reference's repetition of the all-species stencil once per due species.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "gpgmp_oracle.h"

#define IDX(x, y, N) ((size_t)(((y) + (N)) % (N)) * (N) + (size_t)(((x) + (N)) % (N)))

void orc_gs_forward_f32(int N, int steps, float F, float k, float Du, float Dv, float vx, float vy, float dt,
                        float* u, float* v) {
    const size_t n = (size_t)N * N;
    float* u2 = (float*)malloc(sizeof(float) * n);
    float* v2 = (float*)malloc(sizeof(float) * n);
    for (int s = 0; s < steps; ++s) {
        #pragma omp parallel for schedule(static)
        for (int y = 0; y < N; ++y)
            for (int x = 0; x < N; ++x) {
                size_t i = (size_t)y * N + x;
                float uc = u[i], vc = v[i];
                float lu = u[IDX(x - 1, y, N)] + u[IDX(x + 1, y, N)] + u[IDX(x, y - 1, N)] + u[IDX(x, y + 1, N)] - 4.0f * uc;
                float lv = v[IDX(x - 1, y, N)] + v[IDX(x + 1, y, N)] + v[IDX(x, y - 1, N)] + v[IDX(x, y + 1, N)] - 4.0f * vc;
                float uvv = uc * vc * vc;
                float au = vx * (u[IDX(x + 1, y, N)] - u[IDX(x - 1, y, N)]) * 0.5f + vy * (u[IDX(x, y + 1, N)] - u[IDX(x, y - 1, N)]) * 0.5f;
                float av = vx * (v[IDX(x + 1, y, N)] - v[IDX(x - 1, y, N)]) * 0.5f + vy * (v[IDX(x, y + 1, N)] - v[IDX(x, y - 1, N)]) * 0.5f;
                u2[i] = uc + dt * (Du * lu - au - uvv + F * (1.0f - uc));
                v2[i] = vc + dt * (Dv * lv - av + uvv - (F + k) * vc);
            }
        memcpy(u, u2, sizeof(float) * n);
        memcpy(v, v2, sizeof(float) * n);
    }
    free(u2); free(v2);
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

int orc_det_solve(const orc_model* m, float* state, float* snaps, float* snap_times, int max_snaps,
                  int* nsnap, int64_t* steps_out) {
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
        if (m->num_reactions > 0) orc_ref_rk4(m, state, deltat);
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
