/*
 * oracle/orc_rep.c -- TEST INFRASTRUCTURE ONLY (the oracle).
 *
 * CPU replay of this project's CUDA stochastic solver.  The algorithms are those
 * of the reference (direct-method SSA per cell, lattice jumps per species,
 * directionally split drift-diffusion, the oclSolve event loop), drawn from
 * Philox-4x32 streams keyed by (seed, realisation) and counted by
 * (draw, step seed, cell, phase | species | sweep), with jump counts sampled as
 * binomials instead of one uniform per particle.  Same distributions as the
 * reference; bit-identical to the GPU kernels.
 *
 * Reference semantics followed:
 *   SSA window            Gillespie.cl:58-99, hazards Reaction.cpp:119-138
 *   homogeneous jumps     StochasticHomogeneousDiffusion.cl:56-124
 *   source walls          StochasticHomogeneousDiffusion.cl:128-183, HomogeneousSolver.cpp:210-227
 *   drift-diffusion sweep StochasticInhomogeneousDriftDiffusion.cl:505-557, :687-723
 *   per-cell time step    StochasticInhomogeneousDriftDiffusion.cl:124-151
 *   diffusivity / drift   DiffusionModel.cpp:319-380, helpers.cl:18-36
 *   event loop            DiffusionModel.cpp:1414-1603, InhomogeneousSolver.cpp:238-427
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "gpgmp_oracle.h"
#include "orc_math.h"

#define REP_EVENT_CAP (1 << 22)
#define REP_STATUS_EVENT_CAP 1
#define REP_STATUS_OVERFLOW 2

/* ---- initial counts ---------------------------------------------------------- */
void orc_rep_init_poisson(int W, int H, int S, int R, uint32_t seed, const float* lam, int32_t* state) {
    const size_t area = (size_t)W * H;
    #pragma omp parallel for schedule(dynamic, 64) collapse(2)
    for (int r = 0; r < R; ++r)
        for (int64_t c = 0; c < (int64_t)area; ++c) {
            for (int s = 0; s < S; ++s) {
                orc_stream st;
                orc_stream_init(&st, seed, (uint32_t)r, 0u, (uint32_t)c, ORC_PH_INIT | ((uint32_t)s << 8));
                state[((size_t)r * S + s) * area + c] = orc_poisson(&st, lam[s]);
            }
        }
}

/* ---- SSA ------------------------------------------------------------------------ */
static inline float rep_hazard(const orc_reaction* rc, const int32_t* x) {
    float v = rc->rate;
    for (int j = 0; j < rc->num_reactants; ++j) {
        int32_t a = x[rc->reactant_species[j]];
        v = v * (float)a;
        for (int k = 1; k < rc->reactant_stoich[j]; ++k) v = v * (float)(a - k);
    }
    return v;
}

static int rep_apply(const orc_reaction* rc, int32_t* x) {
    for (int j = 0; j < rc->num_products; ++j) {
        int32_t s = rc->product_species[j];
        if (x[s] > INT32_MAX - rc->product_stoich[j]) return REP_STATUS_OVERFLOW;
    }
    for (int j = 0; j < rc->num_reactants; ++j) x[rc->reactant_species[j]] -= rc->reactant_stoich[j];
    for (int j = 0; j < rc->num_products; ++j) x[rc->product_species[j]] += rc->product_stoich[j];
    return 0;
}

/* Custom propensity laws: the product compiles them into its SSA kernel at run time;
 * the replay takes them from the test as a callback (r, counts) -> hazard that
 * evaluates the same float operations.  NULL restores the mass-action hazard. */
typedef float (*orc_hazard_fn)(int r, const int32_t* x);
static orc_hazard_fn g_custom_hazard = NULL;
void orc_set_custom_hazard(orc_hazard_fn fn) { g_custom_hazard = fn; }

/* on: the reactions that may fire in this cell (localised reactions); a reaction that
 * may not has hazard 0 */
static int rep_ssa_cell(const orc_model* m, int32_t* x, orc_stream* st, float window, const uint32_t* on) {
    const int R = m->num_reactions;
    float H[128];
    float t = 0.0f;
    int events = 0;
    for (;;) {
        float h0 = 0.0f;
        for (int r = 0; r < R; ++r) {
            const float hr = !orc_reaction_on(on, r) ? 0.0f
                             : (g_custom_hazard ? g_custom_hazard(r, x) : rep_hazard(&m->reactions[r], x));
            h0 = h0 + hr;
            H[r] = h0;
        }
        if (!(h0 > 0.0f)) break;
        uint32_t a = orc_stream_next(st), b = orc_stream_next(st);
        float r1 = orc_u01_open0(a);
        float r2 = orc_u01(b) * h0;
        float dtev = -orc_logf(r1) / h0;
        t = t + dtev;
        if (!(t < window)) break;
        int j = -1;
        for (int r = 0; r < R; ++r) if (r2 < H[r]) { j = r; break; }
        if (j >= 0) {
            int e = rep_apply(&m->reactions[j], x);
            if (e) return e;
        }
        if (++events >= REP_EVENT_CAP) return REP_STATUS_EVENT_CAP;
    }
    return 0;
}

void orc_rep_ssa(const orc_model* m, int32_t* state, int R, uint32_t seed, uint32_t step_seed, float window,
                 int32_t* status) {
    const int S = m->num_species;
    const size_t area = (size_t)m->width * m->height;
    if (m->num_reactions <= 0) return;
    #pragma omp parallel for schedule(dynamic, 16) collapse(2)
    for (int r = 0; r < R; ++r)
        for (int64_t c = 0; c < (int64_t)area; ++c) {
            int32_t x[64];
            int32_t* base = state + (size_t)r * S * area;
            for (int s = 0; s < S; ++s) x[s] = base[(size_t)s * area + c];
            orc_stream st;
            orc_stream_init(&st, seed, (uint32_t)r, step_seed, (uint32_t)c, ORC_PH_SSA);
            uint32_t on[4];
            orc_cell_reactions(m, (size_t)c, on);
            int e = rep_ssa_cell(m, x, &st, window, on);
            for (int s = 0; s < S; ++s) base[(size_t)s * area + c] = x[s];
            if (e && status) {
                #pragma omp atomic
                status[r] |= e;
            }
        }
}

/* ---- homogeneous jumps --------------------------------------------------------- */
static inline float rep_move_quarter(const orc_model* m) {
    float stay = (float)(1.0 - (double)m->p0);
    return (float)((1.0 - (double)stay) / 6.0);
}

static inline void rep_homog_lost(const orc_model* m, int n, float pmove, orc_stream* st, int x, int y, int l[4]) {
    const int W = m->width, H = m->height;
    l[0] = l[1] = l[2] = l[3] = 0;
    int moved = orc_binomial(st, n, pmove);
    if (moved <= 64) {
        uint32_t w = 0;
        for (int i = 0; i < moved; ++i) {
            if ((i & 15) == 0) w = orc_stream_next(st);
            l[(w >> (2 * (i & 15))) & 3u]++;
        }
    } else {
        l[0] = orc_binomial(st, moved, 0.25f);
        l[1] = orc_binomial(st, moved - l[0], 1.0f / 3.0f);
        l[2] = orc_binomial(st, moved - l[0] - l[1], 0.5f);
        l[3] = moved - l[0] - l[1] - l[2];
    }
    if (x == 0 && m->boundary_mask[0] == 0) l[0] = 0;
    if (x == W - 1 && m->boundary_mask[1] == 0) l[1] = 0;
    if (y == 0 && m->boundary_mask[2] == 0) l[2] = 0;
    if (y == H - 1 && m->boundary_mask[3] == 0) l[3] = 0;
}

static void rep_source(const orc_model* m, int32_t* st_species, uint32_t seed, int r, int species,
                       uint32_t step_seed, int boundary, int source, float pi) {
    const int W = m->width, H = m->height;
    for (int dev = 0; dev < W; ++dev) {
        int gid;
        switch (boundary) {
            case 0: gid = dev * W; break;
            case 1: gid = (W - 1) + dev * W; break;
            case 2: gid = dev; break;
            default: gid = dev + (H - 1) * W; break;
        }
        if (gid >= W * H) continue;
        orc_stream st;
        orc_stream_init(&st, seed, (uint32_t)r, step_seed, (uint32_t)gid,
                        ORC_PH_SOURCE | ((uint32_t)species << 8) | (uint32_t)boundary);
        st_species[gid] += orc_binomial(&st, source, pi);
    }
}

void orc_rep_homog_diffuse(const orc_model* m, int32_t* state, int R, uint32_t seed, int species, uint32_t step_seed) {
    const int W = m->width, H = m->height, S = m->num_species;
    const size_t area = (size_t)W * H;
    const float pi = rep_move_quarter(m);
    const float pmove = pi * 4.0f;
    int32_t* lost = (int32_t*)malloc(sizeof(int32_t) * 4 * area);
    for (int r = 0; r < R; ++r) {
        int32_t* st = state + ((size_t)r * S + species) * area;
        #pragma omp parallel for schedule(static)
        for (int y = 0; y < H; ++y)
            for (int x = 0; x < W; ++x) {
                const int c = x + y * W;
                orc_stream s;
                orc_stream_init(&s, seed, (uint32_t)r, step_seed, (uint32_t)c,
                                ORC_PH_DIFF | ((uint32_t)species << 8));
                rep_homog_lost(m, st[c], pmove, &s, x, y, &lost[4 * c]);
            }
        #pragma omp parallel for schedule(static)
        for (int y = 0; y < H; ++y)
            for (int x = 0; x < W; ++x) {
                const int c = x + y * W;
                int v = st[c] - (lost[4 * c] + lost[4 * c + 1] + lost[4 * c + 2] + lost[4 * c + 3]);
                if (x > 0) v += lost[4 * (c - 1) + 1];
                if (x < W - 1) v += lost[4 * (c + 1) + 0];
                if (y > 0) v += lost[4 * (c - W) + 3];
                if (y < H - 1) v += lost[4 * (c + W) + 2];
                st[c] = v;
            }
        /* HomogeneousSolver.cpp:212-227: wall 0 takes its count from source_mask[1] */
        if (m->source_mask[0] > 0) rep_source(m, st, seed, r, species, step_seed, 0, m->source_mask[1], pi);
        if (m->source_mask[1] > 0) rep_source(m, st, seed, r, species, step_seed, 1, m->source_mask[1], pi);
        if (m->source_mask[2] > 0) rep_source(m, st, seed, r, species, step_seed, 2, m->source_mask[2], pi);
        if (m->source_mask[3] > 0) rep_source(m, st, seed, r, species, step_seed, 3, m->source_mask[3], pi);
    }
    free(lost);
}

/* ---- drift-diffusion sweeps ------------------------------------------------------ */
static inline float rep_clamp01(float v) { return v < 0.0f ? 0.0f : (v > 1.0f ? 1.0f : v); }

static inline void rep_sweep_probs(float D, float r, float dt, float dx, float* Pp, float* Pm) {
    float denom = 2.0f * D + r * r * dt;
    float ps = 1.0f - (dt * denom) / (dx * dx);
    float q = 1.0f - ps;
    float p1 = 0.0f, pm = 0.0f;
    if (denom > 0.0f) {
        float b = (dx * r) / denom;
        p1 = q * (1.0f + b) * 0.5f;
        pm = q * (1.0f - b) * 0.5f;
    }
    *Pp = rep_clamp01(p1);
    float rest = 1.0f - *Pp;
    *Pm = pm < 0.0f ? 0.0f : (pm > rest ? rest : pm);
}

/* stochastic_inhomogeneous_fpe rates (StochasticInhomogeneousDriftDiffusion.cl:197-203)
 * times dt; a negative rate is clamped to 0 */
static inline void rep_sweep_probs_fpe(float D, float r, float dt, float dx, float* Pp, float* Pm) {
    float a = D / (dx * dx), b = r / (2.0f * dx);
    *Pp = rep_clamp01((a + b) * dt);
    float pm = (a - b) * dt, rest = 1.0f - *Pp;
    *Pm = pm < 0.0f ? 0.0f : (pm > rest ? rest : pm);
}

void orc_rep_inhomog_sweep(const orc_model* m, int32_t* state, int R, uint32_t seed, int species, int sweep_y,
                           uint32_t step_seed, float dt, const float* dfield, const float* rfield) {
    const int fpe = m->solver_type == 3;
    const int W = m->width, H = m->height, S = m->num_species;
    const size_t area = (size_t)W * H;
    const float dx = sweep_y ? m->physical_length / (float)H : m->physical_length / (float)W;
    const float* Df = dfield + (size_t)species * area;
    const float* rf = rfield + (size_t)species * area;
    int32_t* lost = (int32_t*)malloc(sizeof(int32_t) * 2 * area);
    for (int r = 0; r < R; ++r) {
        int32_t* st = state + ((size_t)r * S + species) * area;
        #pragma omp parallel for schedule(static)
        for (int y = 0; y < H; ++y)
            for (int x = 0; x < W; ++x) {
                const int c = x + y * W;
                orc_stream s;
                orc_stream_init(&s, seed, (uint32_t)r, step_seed, (uint32_t)c,
                                ORC_PH_DIFF | ((uint32_t)species << 8) | (sweep_y ? 2u : 1u));
                float Pp, Pm;
                if (fpe) rep_sweep_probs_fpe(Df[c], rf[c], dt, dx, &Pp, &Pm);
                else rep_sweep_probs(Df[c], rf[c], dt, dx, &Pp, &Pm);
                float Pt = Pp + Pm;
                int moved = orc_binomial(&s, st[c], Pt);
                int plus = Pt > 0.0f ? orc_binomial(&s, moved, Pp / Pt) : 0;
                int minus = moved - plus;
                int at_lo = sweep_y ? (y == 0) : (x == 0);
                int at_hi = sweep_y ? (y == H - 1) : (x == W - 1);
                if (at_lo && m->boundary_mask[sweep_y ? 2 : 0] == 0) minus = 0;
                if (at_hi && m->boundary_mask[sweep_y ? 3 : 1] == 0) plus = 0;
                lost[2 * c] = minus;
                lost[2 * c + 1] = plus;
            }
        const int stride = sweep_y ? W : 1;
        #pragma omp parallel for schedule(static)
        for (int y = 0; y < H; ++y)
            for (int x = 0; x < W; ++x) {
                const int c = x + y * W;
                int v = st[c] - lost[2 * c] - lost[2 * c + 1];
                int lo = sweep_y ? (y > 0) : (x > 0);
                int hi = sweep_y ? (y < H - 1) : (x < W - 1);
                if (lo) v += lost[2 * (c - stride) + 1];
                if (hi) v += lost[2 * (c + stride)];
                st[c] = v;
            }
    }
    free(lost);
}

float orc_rep_timestep(const orc_model* m, int species, int sweep_y, const float* dfield, const float* rfield) {
    /* StochasticInhomogeneousDriftDiffusion.cl:124-151 per cell (the FPE and deterministic
     * formulas by solver type), then the minimum (:382-423) */
    const size_t area = (size_t)m->width * m->height;
    const float dx = m->physical_length / (float)m->width;
    const float* Df = dfield + (size_t)species * area;
    const float* rf = rfield + (size_t)species * area;
    (void)sweep_y;
    const int ty = m->solver_type;
    const float stay = (float)(1.0 - (double)m->p0);
    float best = INFINITY;
    for (size_t c = 0; c < area; ++c) {
        float ts = ty == 3 ? orc_fpe_timestep(Df[c], rf[c], dx, stay)
                 : (ty == 5 || ty == 6) ? orc_det_timestep(Df[c], rf[c], dx)
                 : orc_cell_timestep(Df[c], rf[c], dx);
        if (ts == ts) best = fminf(best, ts);
    }
    return best;
}

/* DiffusionModel.cpp:319-380 built-in methods; PhysicalX as helpers.cl:29-36. */
void orc_rep_diffusivity_drift(const orc_model* m, int species, float* dx, float* dy, float* rx, float* ry) {
    const int W = m->width, H = m->height;
    const size_t area = (size_t)W * H, off = (size_t)species * area;
    const float L = m->physical_length;
    const float* p = m->drift_params;
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            size_t i = off + (size_t)x + (size_t)y * W;
            float px = L / (float)W * ((float)x - (float)W * 0.5f);
            float py = L / (float)H * ((float)y - (float)H * 0.5f);
            switch (m->drift_method) {
                case 0: dx[i] = p[0]; dy[i] = p[1]; rx[i] = p[2]; ry[i] = p[3]; break;
                case 1: {
                    float sx = px + L, sy = py + L;
                    dx[i] = (p[0] * p[0]) * (sx * sx) * 0.5f;
                    dy[i] = (p[1] * p[1]) * (sy * sy) * 0.5f;
                    rx[i] = p[2] * sx;
                    ry[i] = p[3] * sy;
                    break;
                }
                case 2:
                    dx[i] = p[0]; dy[i] = p[1];
                    rx[i] = -(p[2] * px + p[3] * py);
                    ry[i] = -(p[4] * px + p[5] * py);
                    break;
                default:
                    dx[i] = m->field_dx ? m->field_dx[i] : 0.0f;
                    dy[i] = m->field_dy ? m->field_dy[i] : 0.0f;
                    rx[i] = m->field_rx ? m->field_rx[i] : 0.0f;
                    ry[i] = m->field_ry ? m->field_ry[i] : 0.0f;
                    break;
            }
        }
}

/* ---- event loop ---------------------------------------------------------------- */
static int any_status(const int32_t* st, int R) {
    if (!st) return 0;
    for (int r = 0; r < R; ++r) if (st[r]) return 1;
    return 0;
}

int orc_rep_solve(const orc_model* m, int32_t* state, int R, uint32_t seed,
                  int32_t* snaps, float* snap_times, int max_snaps, int* nsnap,
                  int64_t* steps_out, int32_t* status) {
    const int S = m->num_species;
    const size_t area = (size_t)m->width * m->height;
    const size_t block = (size_t)R * S * area;
    const int inhom = m->solver_type == 1 || m->solver_type == 3;
    const int stop_on_error = (m->flags & 4) != 0;
    const float h = m->physical_length / (float)m->width;
    float* dtv = (float*)calloc(S, sizeof(float));
    float* next = (float*)calloc(S, sizeof(float));
    float *nx = NULL, *ny = NULL, *sdx = NULL, *sdy = NULL, *ddx = NULL, *ddy = NULL;
    float *Fdx = NULL, *Fdy = NULL, *Frx = NULL, *Fry = NULL;
    if (!inhom) {
        for (int i = 0; i < S; ++i) {
            dtv[i] = m->diffusion[i] > 0 ? m->p0 / ((float)2. * 3) * h * h / m->diffusion[i] : m->max_time;
            next[i] = dtv[i];
        }
    } else {
        nx = (float*)calloc(S, sizeof(float)); ny = (float*)calloc(S, sizeof(float));
        sdx = (float*)calloc(S, sizeof(float)); sdy = (float*)calloc(S, sizeof(float));
        ddx = (float*)calloc(S, sizeof(float)); ddy = (float*)calloc(S, sizeof(float));
        Fdx = (float*)malloc(sizeof(float) * S * area); Fdy = (float*)malloc(sizeof(float) * S * area);
        Frx = (float*)malloc(sizeof(float) * S * area); Fry = (float*)malloc(sizeof(float) * S * area);
        for (int i = 0; i < S; ++i) {
            orc_rep_diffusivity_drift(m, i, Fdx, Fdy, Frx, Fry);
            sdx[i] = orc_rep_timestep(m, i, 0, Fdx, Frx);
            sdy[i] = orc_rep_timestep(m, i, 1, Fdy, Fry);
            ddx[i] = sdx[i]; ddy[i] = sdy[i];
            nx[i] = sdx[i]; ny[i] = sdy[i];
        }
        for (int i = 0; i < S; ++i) next[i] = nx[i] < ny[i] ? nx[i] : ny[i];
    }
    int ns = 0;
#define SNAP(t) do { if (ns < max_snaps) { memcpy(snaps + (size_t)ns * block, state, sizeof(int32_t) * block); \
                      snap_times[ns] = (t); } ns++; } while (0)
    SNAP(0.f);
    float simTime = 0.f, outputLast = 0.f;
    int64_t n = 0;
    while ((m->max_steps < 0 || n < m->max_steps) && simTime < m->max_time) {
        uint32_t sd = (uint32_t)n * 64u;
        n++;
        float mindt = next[0];
        int minspec = 0;
        for (int i = 1; i < S; ++i) if (next[i] < mindt) { mindt = next[i]; minspec = i; }
        int ev = 0;
        float mo = outputLast + m->output_interval;
        if (mo < mindt) { mindt = mo; ev = 1; }
        float deltat = mindt - simTime;
        if (m->num_reactions > 0) { orc_rep_ssa(m, state, R, seed, sd, deltat, status); sd++; }
        if (ev == 0) {
            for (int i = 0; i < S; ++i) {
                if (!(i == minspec || next[i] <= mindt)) continue;
                if (!(next[i] > 0)) continue;
                if (!inhom) {
                    orc_rep_homog_diffuse(m, state, R, seed, i, sd);
                    next[i] += dtv[i];
                } else {
                    if (nx[i] <= mindt) {
                        orc_rep_inhomog_sweep(m, state, R, seed, i, 0, sd, ddx[i], Fdx, Frx);
                        sd++;
                        nx[i] += sdx[i];
                        ddx[i] = sdx[i];
                    }
                    if (ny[i] <= mindt) {
                        orc_rep_inhomog_sweep(m, state, R, seed, i, 1, sd, ddy[i], Fdy, Fry);
                        sd++;
                        ny[i] += sdy[i];
                        ddy[i] = sdy[i];
                    }
                }
            }
            if (inhom) for (int i = 0; i < S; ++i) next[i] = nx[i] < ny[i] ? nx[i] : ny[i];
        } else {
            if (simTime >= outputLast + m->output_interval) {
                SNAP(mindt);
                outputLast += m->output_interval;
            }
        }
        simTime = mindt;
        if (stop_on_error && any_status(status, R)) break;
    }
    SNAP(simTime);
#undef SNAP
    *nsnap = ns;
    *steps_out = n;
    free(dtv); free(next);
    free(nx); free(ny); free(sdx); free(sdy); free(ddx); free(ddy);
    free(Fdx); free(Fdy); free(Frx); free(Fry);
    return 0;
}

/* ---- individual species ------------------------------------------------------------
 * One sweep of an individual species with the properties as stored (no model code),
 * restating individual_device.cuh (ind_sweep_body, ind_counts_body) after the
 * reference's individual_diffuseX/Y and computeDiffusionConstants
 * (IndividualSolver.cl:654-1015): every individual draws once (stream (seed, r),
 * counter (step_seed, id, PH_INDIV | species << 8 | dir)) and moves one cell with the
 * inhomogeneous sweep's probabilities of its own D and r; reflecting walls cancel the
 * move, absorbing walls remove it (key = R * area).  Then the counts of the species'
 * planes and the fields [4][R*area] (largest D x, D y, |r x|, |r y| of the individuals
 * in each cell).  keys are updated in place and not sorted (orc_rep_ind_sort sorts);
 * returns the number that left in this sweep. */
int64_t orc_rep_ind_sweep(const orc_model* m, int32_t* state, int R, uint32_t seed, int species, int dir, float dt,
                          uint32_t step_seed, uint32_t* keys, const uint32_t* ids, int64_t n, const float* props,
                          int64_t cap, float* fields) {
    const int W = m->width, H = m->height, S = m->num_species;
    const int64_t area = (int64_t)W * H, ncells = area * R;
    const float dx = m->physical_length / (float)(dir == 0 ? W : H);
    const uint32_t killed = (uint32_t)ncells;
    int64_t left = 0;
    for (int64_t k = 0; k < 4 * ncells; ++k) fields[k] = 0.f;
    for (int64_t k = 0; k < ncells; ++k) {
        const int r = (int)(k / area);
        state[((int64_t)r * S + species) * area + (k - (int64_t)r * area)] = 0;
    }
    for (int64_t i = 0; i < n; ++i) {
        const uint32_t key = keys[i], id = ids[i];
        if (key >= killed) continue;
        const int r = (int)(key / area);
        const int cell = (int)(key - (int64_t)r * area);
        const int gx = cell % W, gy = cell / W;
        const float D = props[(dir == 0 ? 0 : 1) * cap + id];
        const float v = props[(dir == 0 ? 2 : 3) * cap + id];
        float Pp, Pm;
        rep_sweep_probs(D, v, dt, dx, &Pp, &Pm);
        orc_stream s;
        orc_stream_init(&s, seed, (uint32_t)r, step_seed, id, ORC_PH_INDIV | ((uint32_t)species << 8) | (uint32_t)dir);
        const float u = orc_u01(orc_stream_next(&s));
        const int mv = u < Pp ? 1 : (u < Pp + Pm ? -1 : 0);
        uint32_t out = key;
        if (mv != 0) {
            const int c = dir == 0 ? gx : gy, lim = dir == 0 ? W : H, nc = c + mv;
            if (nc < 0 || nc >= lim) {
                const int wall = (dir == 0 ? 0 : 2) + (mv > 0 ? 1 : 0);
                if (m->boundary_mask[wall] != 0) out = killed;
            } else {
                out = (uint32_t)((int64_t)r * area + (dir == 0 ? gy * W + nc : nc * W + gx));
            }
            keys[i] = out;
        }
        if (out >= killed) { ++left; continue; }
        state[((int64_t)r * S + species) * area + (out - (int64_t)r * area)] += 1;
        fields[out] = fmaxf(fields[out], props[id]);
        fields[ncells + out] = fmaxf(fields[ncells + out], props[cap + id]);
        fields[2 * ncells + out] = fmaxf(fields[2 * ncells + out], fabsf(props[2 * cap + id]));
        fields[3 * ncells + out] = fmaxf(fields[3 * ncells + out], fabsf(props[3 * cap + id]));
    }
    return left;
}

/* the list in key order (a stable sort), the individuals that left (key ncells) taken
 * out: their ids are written to killed_ids; returns the remaining length */
int64_t orc_rep_ind_sort(uint32_t* keys, uint32_t* ids, int64_t n, int64_t ncells, uint32_t* killed_ids,
                         int64_t* n_killed) {
    int64_t* cnt = (int64_t*)calloc((size_t)ncells + 2, sizeof(int64_t));
    uint32_t* k2 = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)(n > 0 ? n : 1));
    uint32_t* i2 = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)(n > 0 ? n : 1));
    for (int64_t i = 0; i < n; ++i) cnt[keys[i] + 1]++;
    for (int64_t b = 0; b <= ncells; ++b) cnt[b + 1] += cnt[b];
    for (int64_t i = 0; i < n; ++i) {
        int64_t o = cnt[keys[i]]++;
        k2[o] = keys[i];
        i2[o] = ids[i];
    }
    int64_t alive = 0, nk = 0;
    for (int64_t i = 0; i < n; ++i) {
        if (k2[i] >= (uint32_t)ncells) killed_ids[nk++] = i2[i];
        else { keys[alive] = k2[i]; ids[alive] = i2[i]; ++alive; }
    }
    *n_killed = nk;
    free(cnt); free(k2); free(i2);
    return alive;
}

/* the smallest time step over n cells of fields D, r (the stochastic formula) */
float orc_rep_timestep_cells(const float* D, const float* r, int64_t n, float dx) {
    float best = INFINITY;
    for (int64_t c = 0; c < n; ++c) {
        float ts = orc_cell_timestep(D[c], r[c], dx);
        if (ts == ts) best = fminf(best, ts);
    }
    return best;
}
