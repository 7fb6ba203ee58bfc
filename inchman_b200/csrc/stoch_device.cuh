// Per-cell device routines of the stochastic solvers, shared by the wide kernels
// (one launch covers every realisation) and the persistent ensemble kernel.
//
// Reference semantics (paths inside the reference project):
//   ssa_cell      Gillespie.cl:58-99 direct method; hazards Reaction.cpp:119-138;
//                 reaction picked where the cumulative hazard first exceeds r2,
//                 which is what the isless/isgreaterequal masks of
//                 Solver.cpp:865-904 select; the event that crosses the window
//                 end is discarded (Gillespie.cl:80).
//   homog_lost    StochasticHomogeneousDiffusion.cl:56-92: each particle moves to
//                 one of four neighbours with probability (1-Stay)/6 each;
//                 reflecting walls keep it, absorbing walls lose it.  Here the
//                 four counts are one multinomial draw (binomial for "moved",
//                 then an equal four-way split) instead of one uniform per particle.
//   sweep_probs   StochasticInhomogeneousDriftDiffusion.cl:512-520 (X) and
//                 :642-650 (Y): ps, p1 (towards +), p2-p1 (towards -).
//   cell_timestep StochasticInhomogeneousDriftDiffusion.cl:124-151 (and the FPE
//                 and deterministic variants of the same kernel).
#pragma once
#include "common.cuh"
#include "../../include/gpgmp_c.h"

namespace gpgmp {

__device__ __forceinline__ float hazard(const gpgmp_reaction& rc, const int* x, int stride) {
    float v = rc.rate;
    for (int j = 0; j < rc.num_reactants; ++j) {
        const int a = x[rc.reactant_species[j] * stride];
        v = v * (float)a;
        for (int k = 1; k < rc.reactant_stoich[j]; ++k) v = v * (float)(a - k);
    }
    return v;
}

// The mass-action hazard as a functor; a model with custom propensity laws supplies
// its own (compiled at run time, csrc/jit.cpp).
struct MassActionHazard {
    __device__ __forceinline__ float operator()(const gpgmp_reaction* rt, int r, const int* x, int stride) const {
        return hazard(rt[r], x, stride);
    }
};

// Localised reactions: bit r of on[r / 32] says whether reaction r may fire in this
// cell (Reaction::reactionMask, Reaction.cpp:216-235).  The reference multiplies the
// law by the mask value 1 or 0 (Solver.cpp:852-854); a zero hazard is the same sum.
struct CellReactions {
    uint32_t on[4];
    // rmask: [words][area] bits of the cells (words = ceil(reactions / 32)); NULL: all on
    __device__ __forceinline__ void load(const uint32_t* __restrict__ rmask, int words, int area, int c) {
        on[0] = on[1] = on[2] = on[3] = 0xFFFFFFFFu;
        if (rmask)
            for (int w = 0; w < words; ++w) on[w] = rmask[(int64_t)w * area + c];
    }
    __device__ __forceinline__ bool operator()(int r) const { return (on[r >> 5] >> (r & 31)) & 1u; }
};
struct AllReactions {
    __device__ __forceinline__ bool operator()(int) const { return true; }
};
template <class HZ>
struct GatedHazard {
    HZ hz;
    CellReactions on;
    __device__ __forceinline__ float operator()(const gpgmp_reaction* rt, int r, const int* x, int stride) const {
        return on(r) ? hz(rt, r, x, stride) : 0.0f;
    }
};

// Runs one SSA window on the counts x[s * stride]; returns a GPGMP_SIM_* bit or 0.
template <class HZ>
__device__ __forceinline__ int ssa_cell_h(const gpgmp_reaction* rt, int R, int* x, int stride, Stream& st,
                                          float window, const HZ& hz) {
    float t = 0.0f;
    int events = 0;
    for (;;) {
        float h0 = 0.0f;
        for (int r = 0; r < R; ++r) h0 = h0 + hz(rt, r, x, stride);
        if (!(h0 > 0.0f)) return 0;
        const uint32_t a = st.next(), b = st.next();
        const float r1 = u01_open0(a);
        const float r2 = u01(b) * h0;
        const float dtev = -gp_logf(r1) / h0;
        t = t + dtev;
        if (!(t < window)) return 0;
        // second pass: same partial sums, stop at the first one above r2
        int j = -1;
        float hc = 0.0f;
        for (int r = 0; r < R; ++r) {
            hc = hc + hz(rt, r, x, stride);
            if (r2 < hc) { j = r; break; }
        }
        if (j >= 0) {
            const gpgmp_reaction& rc = rt[j];
            for (int q = 0; q < rc.num_products; ++q)
                if (x[rc.product_species[q] * stride] > INT32_MAX - rc.product_stoich[q]) return SIM_OVERFLOW;
            for (int q = 0; q < rc.num_reactants; ++q) x[rc.reactant_species[q] * stride] -= rc.reactant_stoich[q];
            for (int q = 0; q < rc.num_products; ++q) x[rc.product_species[q] * stride] += rc.product_stoich[q];
        }
        if (++events >= SSA_EVENT_CAP) return SIM_EVENT_CAP;
    }
}
__device__ __forceinline__ int ssa_cell(const gpgmp_reaction* rt, int R, int* x, int stride, Stream& st,
                                        float window) {
    return ssa_cell_h(rt, R, x, stride, st, window, MassActionHazard{});
}

// Dependency masks of the incremental SSA: bit q of deps[j * 4 + q / 32] is set when
// reaction j changes the count of a species that reaction q consumes, i.e. when q's
// hazard must be recomputed after j fires (Gibson & Bruck's dependency graph).  Built
// by all threads of a block; R <= 128.
__device__ __forceinline__ void build_deps(const gpgmp_reaction* rt, int R, uint32_t* deps) {
    for (int idx = threadIdx.x; idx < R * 4; idx += blockDim.x) deps[idx] = 0u;
    __syncthreads();
    for (int idx = threadIdx.x; idx < R * R; idx += blockDim.x) {
        const int j = idx / R, q = idx % R;
        const gpgmp_reaction& a = rt[j];
        const gpgmp_reaction& b = rt[q];
        bool dep = false;
        for (int u = 0; u < b.num_reactants && !dep; ++u) {
            const int sp = b.reactant_species[u];
            int net = 0;
            for (int v = 0; v < a.num_reactants; ++v) if (a.reactant_species[v] == sp) net -= a.reactant_stoich[v];
            for (int v = 0; v < a.num_products; ++v) if (a.product_species[v] == sp) net += a.product_stoich[v];
            dep = net != 0;
        }
        if (dep) atomicOr(&deps[j * 4 + (q >> 5)], 1u << (q & 31));
    }
    __syncthreads();
}

// The same SSA window as ssa_cell with per-reaction hazards kept in h[r * stride]
// and recomputed only where the fired reaction changed a reactant count.  The total
// and the selection sum the same values in the same order as the full recomputation,
// so the result is bit-identical.
// ON(r) gates the reactions of localised models (CellReactions), as in ssa_cell_h.
template <class ON = AllReactions>
__device__ __forceinline__ int ssa_cell_inc(const gpgmp_reaction* rt, const uint32_t* deps, int R, int* x, int stride,
                                            float* h, Stream& st, float window, const ON& on = ON{}) {
    for (int r = 0; r < R; ++r) h[r * stride] = on(r) ? hazard(rt[r], x, stride) : 0.0f;
    float t = 0.0f;
    int events = 0;
    for (;;) {
        float h0 = 0.0f;
        for (int r = 0; r < R; ++r) h0 = h0 + h[r * stride];
        if (!(h0 > 0.0f)) return 0;
        const uint32_t a = st.next(), b = st.next();
        const float r1 = u01_open0(a);
        const float r2 = u01(b) * h0;
        const float dtev = -gp_logf(r1) / h0;
        t = t + dtev;
        if (!(t < window)) return 0;
        int j = -1;
        float hc = 0.0f;
        for (int r = 0; r < R; ++r) {
            hc = hc + h[r * stride];
            if (r2 < hc) { j = r; break; }
        }
        if (j >= 0) {
            const gpgmp_reaction& rc = rt[j];
            for (int q = 0; q < rc.num_products; ++q)
                if (x[rc.product_species[q] * stride] > INT32_MAX - rc.product_stoich[q]) return SIM_OVERFLOW;
            for (int q = 0; q < rc.num_reactants; ++q) x[rc.reactant_species[q] * stride] -= rc.reactant_stoich[q];
            for (int q = 0; q < rc.num_products; ++q) x[rc.product_species[q] * stride] += rc.product_stoich[q];
            for (int w = 0; w * 32 < R; ++w) {
                uint32_t m = deps[j * 4 + w];
                while (m) {
                    const int q = w * 32 + __ffs(m) - 1;
                    m &= m - 1;
                    h[q * stride] = on(q) ? hazard(rt[q], x, stride) : 0.0f;
                }
            }
        }
        if (++events >= SSA_EVENT_CAP) return SIM_EVENT_CAP;
    }
}

// Four lost counts (-x, +x, -y, +y) of one cell of n particles.
__device__ __forceinline__ void homog_lost(int n, float pmove, Stream& st, int x, int y, int W, int H,
                                           const int* bmask, int l[4]) {
    l[0] = l[1] = l[2] = l[3] = 0;
    const int moved = binomial(st, n, pmove);
    if (moved <= 64) {
        uint32_t w = 0;
        for (int i = 0; i < moved; ++i) {
            if ((i & 15) == 0) w = st.next();
            const uint32_t d = (w >> (2 * (i & 15))) & 3u;
            l[0] += d == 0u; l[1] += d == 1u; l[2] += d == 2u; l[3] += d == 3u;
        }
    } else {
        l[0] = binomial(st, moved, 0.25f);
        l[1] = binomial(st, moved - l[0], 1.0f / 3.0f);
        l[2] = binomial(st, moved - l[0] - l[1], 0.5f);
        l[3] = moved - l[0] - l[1] - l[2];
    }
    if (x == 0 && bmask[0] == 0) l[0] = 0;
    if (x == W - 1 && bmask[1] == 0) l[1] = 0;
    if (y == 0 && bmask[2] == 0) l[2] = 0;
    if (y == H - 1 && bmask[3] == 0) l[3] = 0;
}

__device__ __forceinline__ float clamp01(float v) { return v < 0.0f ? 0.0f : (v > 1.0f ? 1.0f : v); }

__device__ __forceinline__ void sweep_probs(float D, float r, float dt, float dx, float* Pp, float* Pm) {
    const float denom = 2.0f * D + r * r * dt;
    const float ps = 1.0f - (dt * denom) / (dx * dx);
    const float q = 1.0f - ps;
    float p1 = 0.0f, pm = 0.0f;
    if (denom > 0.0f) {
        const float b = (dx * r) / denom;
        p1 = q * (1.0f + b) * 0.5f;
        pm = q * (1.0f - b) * 0.5f;
    }
    *Pp = clamp01(p1);
    const float rest = 1.0f - *Pp;
    *Pm = pm < 0.0f ? 0.0f : (pm > rest ? rest : pm);
}

// The FPE discretisation's jump probabilities (stochastic_inhomogeneous_fpe,
// StochasticInhomogeneousDriftDiffusion.cl:197-203 rates, :493-499 use): rate
// towards + is D/dx^2 + r/(2 dx), towards - is D/dx^2 - r/(2 dx), times dt.  A rate
// that comes out negative (|r| dx > 2 D) is clamped to 0.
__device__ __forceinline__ void sweep_probs_fpe(float D, float r, float dt, float dx, float* Pp, float* Pm) {
    const float a = D / (dx * dx), b = r / (2.0f * dx);
    *Pp = clamp01((a + b) * dt);
    const float pm = (a - b) * dt, rest = 1.0f - *Pp;
    *Pm = pm < 0.0f ? 0.0f : (pm > rest ? rest : pm);
}

// (minus, plus) counts of one cell for a directional sweep.
__device__ __forceinline__ void sweep_lost(int n, float D, float r, float dt, float dx, Stream& st, bool at_lo,
                                           bool at_hi, int mask_lo, int mask_hi, int* minus, int* plus,
                                           bool fpe = false) {
    float Pp, Pm;
    if (fpe)
        sweep_probs_fpe(D, r, dt, dx, &Pp, &Pm);
    else
        sweep_probs(D, r, dt, dx, &Pp, &Pm);
    const float Pt = Pp + Pm;
    const int moved = binomial(st, n, Pt);
    int p = Pt > 0.0f ? binomial(st, moved, Pp / Pt) : 0;
    int m = moved - p;
    if (at_lo && mask_lo == 0) m = 0;
    if (at_hi && mask_hi == 0) p = 0;
    *minus = m;
    *plus = p;
}

// Evaluated in double; below |eps| = 1e-3 tanh and temp come from their series
// (tanh eps = eps - eps^3/3, temp = 1/3 + 4 eps^2/45) because the closed form
// cancels there (in float it gives NaN or 0 for small drift).
__device__ __forceinline__ double cell_timestep_d(float Df, float rf, float dxf) {
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
        const double t = gp_exp_d(-2.0 * a);
        const double tha = (1.0 - t) / (1.0 + t);
        th = eps < 0.0 ? -tha : tha;
        const double E = gp_exp_d(a);
        const double sha = (E - 1.0 / E) * 0.5;
        temp = 1.0 + (-1.0 / (th * eps) + 1.0 / (sha * sha));
        if (temp <= 0.0) temp = 1.0 / 3.0;
    }
    return dx / r * th * temp;
}
__device__ __forceinline__ float cell_timestep(float D, float r, float dx) { return (float)cell_timestep_d(D, r, dx); }

// Time step kinds of the per-cell minimum (StochasticInhomogeneousDriftDiffusion.cl:
// 124-151 stochastic, :124-129 FPE, :157-190 deterministic RK4 / alpha-QSS).
enum TimestepKind { kTsStochastic = 0, kTsFpe = 1, kTsDeterministic = 2 };

// FPE: StayProbability / 6 / (D / dx^2 + |r| / (2 dx)), in float.
__device__ __forceinline__ float fpe_timestep(float D, float r, float dx, float stay) {
    return stay / 6.0f / (D / (dx * dx) + fabsf(r) / (2.0f * dx));
}

// deterministic inhomogeneous solvers: the stochastic formula scaled by 0.1 where
// there is drift (the reference's r == 0 branch is not scaled); with D = 0 the
// reference divides by zero, here the step is 0.1 dx / |r|.
__device__ __forceinline__ float det_timestep(float D, float r, float dx) {
    if (r == 0.0f) return (float)cell_timestep_d(D, r, dx);
    return (float)(0.1 * cell_timestep_d(D, r, dx));
}

}  // namespace gpgmp
