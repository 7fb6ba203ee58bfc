// Wide kernels of the stochastic and reference-compatible deterministic solvers.
// One launch covers every realisation of a solver (grid z or the flattened
// index runs over realisations); the host event loop drives them.
//
// Compiled with -fmad=false: the sampling code must round exactly as its CPU
// replay does.
#include <cstdio>
#include "kernels.h"
#include "stoch_device.cuh"

namespace gpgmp {

namespace {

constexpr int kIncMinReactions = 6;   // networks above this size keep per-reaction hazards
constexpr int NT = 256;               // threads of a diffusion tile block

// Launch shapes the autotuner chooses from (GridDesc::tile, GridDesc::ssa_threads):
// diffusion tiles of TW x TH cells for 256 threads (1, 2 or 4 cells per thread in the
// gather; the one-cell halo is recomputed, so wider tiles recompute less), and SSA
// blocks of 64, 128 or 256 threads (one cell per thread).  Every draw is keyed by its
// cell, so all shapes give the same bits.
constexpr int kTileW[kNumDiffusionTiles] = {32, 32, 64, 16, 64, 32};
constexpr int kTileH[kNumDiffusionTiles] = {16, 8, 8, 16, 16, 32};
constexpr int kSsaThreadChoices[kNumSsaThreadChoices] = {128, 64, 256};

__global__ void k_init_poisson(Planes planes, int S, int area, int R, uint32_t seed, const float* __restrict__ lam) {
    const int64_t total = (int64_t)R * area;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int r = (int)(i / area);
        const int c = (int)(i - (int64_t)r * area);
        for (int s = 0; s < S; ++s) {
            Stream st;
            st.init(seed, (uint32_t)r, 0u, (uint32_t)c, PH_INIT | ((uint32_t)s << 8));
            planes.p[s][((int64_t)r * S + s) * area + c] = poisson(st, lam[s]);
        }
    }
}

// MASKED: localised reactions, rmask as GridDesc::rmask (the unmasked form is the
// same code with every reaction on)
template <bool MASKED, int kSsaThreads>
__global__ void __launch_bounds__(kSsaThreads) k_ssa(Planes planes, int S, int area, int R,
                                                     const gpgmp_reaction* __restrict__ reactions, int nreac,
                                                     uint32_t seed, uint32_t step_seed, float window,
                                                     int32_t* __restrict__ status,
                                                     const uint32_t* __restrict__ rmask, int rmask_words) {
    extern __shared__ __align__(16) unsigned char smem[];
    gpgmp_reaction* rt = reinterpret_cast<gpgmp_reaction*>(smem);
    uint32_t* deps = reinterpret_cast<uint32_t*>(smem + sizeof(gpgmp_reaction) * nreac);
    float* hs = reinterpret_cast<float*>(deps + 4 * nreac);
    int* xs = reinterpret_cast<int*>(hs + (size_t)nreac * kSsaThreads);
    for (int i = threadIdx.x; i < nreac; i += blockDim.x) rt[i] = reactions[i];
    __syncthreads();
    build_deps(rt, nreac, deps);
    const int64_t total = (int64_t)R * area;
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= total) return;
    const int r = (int)(i / area);
    const int c = (int)(i - (int64_t)r * area);
    int* x = xs + threadIdx.x;
    for (int s = 0; s < S; ++s) x[s * kSsaThreads] = planes.p[s][((int64_t)r * S + s) * area + c];
    Stream st;
    st.init(seed, (uint32_t)r, step_seed, (uint32_t)c, PH_SSA);
    // both forms give the same bits; the incremental one pays off for larger networks
    int e;
    if (MASKED) {
        CellReactions on;
        on.load(rmask, rmask_words, area, c);
        e = nreac > kIncMinReactions ? ssa_cell_inc(rt, deps, nreac, x, kSsaThreads, hs + threadIdx.x, st, window, on)
                                     : ssa_cell_h(rt, nreac, x, kSsaThreads, st, window,
                                                  GatedHazard<MassActionHazard>{MassActionHazard{}, on});
    } else {
        e = nreac > kIncMinReactions ? ssa_cell_inc(rt, deps, nreac, x, kSsaThreads, hs + threadIdx.x, st, window)
                                     : ssa_cell(rt, nreac, x, kSsaThreads, st, window);
    }
    for (int s = 0; s < S; ++s) planes.p[s][((int64_t)r * S + s) * area + c] = x[s * kSsaThreads];
    if (e) atomicOr(&status[r], e);
}

// MODE 0: 2-D homogeneous jumps; 1: drift-diffusion sweep in x; 2: sweep in y.
// A block owns a TW x TH tile, samples the lost counts of the tile and of its
// one-cell halo (recomputed, the streams are keyed by cell) into shared memory,
// then gathers.  Reads `in`, writes `out`: no block reads what another writes.
template <int MODE, int TW, int TH>
__global__ void __launch_bounds__(NT) k_diffuse_tile(const int* __restrict__ in, int* __restrict__ out, int W, int H,
                                                     int S, int species, uint32_t seed, uint32_t step_seed,
                                                     float pmove, int4 bm4, const float* __restrict__ Df,
                                                     const float* __restrict__ rf, float dt, float dx, int fpe) {
    constexpr int HX = (MODE == 2) ? 0 : 1;
    constexpr int HY = (MODE == 1) ? 0 : 1;
    constexpr int RW = TW + 2 * HX, RH = TH + 2 * HY;
    constexpr int NL = (MODE == 0) ? 4 : 2;
    __shared__ int s_lost[RH * RW * NL];
    __shared__ int s_n[TH * TW];
    const int area = W * H;
    const int r = blockIdx.z;
    const int x0 = blockIdx.x * TW, y0 = blockIdx.y * TH;
    const int64_t plane = ((int64_t)r * S + species) * area;
    const int bm[4] = {bm4.x, bm4.y, bm4.z, bm4.w};
    const uint32_t phase = PH_DIFF | ((uint32_t)species << 8) | (uint32_t)MODE;
    for (int i = threadIdx.x; i < RW * RH; i += NT) {
        const int lx = i % RW, ly = i / RW;
        const int gx = x0 + lx - HX, gy = y0 + ly - HY;
        int l[4] = {0, 0, 0, 0};
        if (gx >= 0 && gx < W && gy >= 0 && gy < H) {
            const int c = gy * W + gx;
            const int n = in[plane + c];
            Stream st;
            st.init(seed, (uint32_t)r, step_seed, (uint32_t)c, phase);
            if (MODE == 0) {
                homog_lost(n, pmove, st, gx, gy, W, H, bm, l);
            } else if (MODE == 1) {
                const int64_t fi = (int64_t)species * area + c;
                sweep_lost(n, Df[fi], rf[fi], dt, dx, st, gx == 0, gx == W - 1, bm[0], bm[1], &l[0], &l[1],
                           fpe != 0);
            } else {
                const int64_t fi = (int64_t)species * area + c;
                sweep_lost(n, Df[fi], rf[fi], dt, dx, st, gy == 0, gy == H - 1, bm[2], bm[3], &l[0], &l[1],
                           fpe != 0);
            }
            if (lx >= HX && lx < HX + TW && ly >= HY && ly < HY + TH) s_n[(ly - HY) * TW + (lx - HX)] = n;
        }
#pragma unroll
        for (int d = 0; d < NL; ++d) s_lost[i * NL + d] = l[d];
    }
    __syncthreads();
    for (int i = threadIdx.x; i < TW * TH; i += NT) {
        const int lx = i % TW, ly = i / TW;
        const int gx = x0 + lx, gy = y0 + ly;
        if (gx >= W || gy >= H) continue;
        const int o = (ly + HY) * RW + (lx + HX);
        int v = s_n[i];
        if (MODE == 0) {
            v -= s_lost[o * 4] + s_lost[o * 4 + 1] + s_lost[o * 4 + 2] + s_lost[o * 4 + 3];
            if (gx > 0) v += s_lost[(o - 1) * 4 + 1];
            if (gx < W - 1) v += s_lost[(o + 1) * 4 + 0];
            if (gy > 0) v += s_lost[(o - RW) * 4 + 3];
            if (gy < H - 1) v += s_lost[(o + RW) * 4 + 2];
        } else if (MODE == 1) {
            v -= s_lost[o * 2] + s_lost[o * 2 + 1];
            if (gx > 0) v += s_lost[(o - 1) * 2 + 1];
            if (gx < W - 1) v += s_lost[(o + 1) * 2];
        } else {
            v -= s_lost[o * 2] + s_lost[o * 2 + 1];
            if (gy > 0) v += s_lost[(o - RW) * 2 + 1];
            if (gy < H - 1) v += s_lost[(o + RW) * 2];
        }
        out[plane + gy * W + gx] = v;
    }
}

__global__ void k_source(int* plane_base, int W, int H, int S, int R, int species, uint32_t seed,
                         uint32_t step_seed, int boundary, int count, float pi) {
    const int total = R * W;
    const int area = W * H;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        const int r = i / W, dev = i % W;
        int gid;
        switch (boundary) {
            case 0: gid = dev * W; break;
            case 1: gid = (W - 1) + dev * W; break;
            case 2: gid = dev; break;
            default: gid = dev + (H - 1) * W; break;
        }
        if (gid >= area) continue;
        Stream st;
        st.init(seed, (uint32_t)r, step_seed, (uint32_t)gid,
                PH_SOURCE | ((uint32_t)species << 8) | (uint32_t)boundary);
        plane_base[((int64_t)r * S + species) * area + gid] += binomial(st, count, pi);
    }
}

__device__ __forceinline__ uint32_t float_key(float f) {
    const uint32_t b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

__global__ void k_timestep(int area, const float* __restrict__ D, const float* __restrict__ r, float dx,
                           uint32_t* min_key, int kind, float stay) {
    uint32_t best = 0xffffffffu;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < area; c += gridDim.x * blockDim.x)
    {
        const float ts = kind == kTsFpe             ? fpe_timestep(D[c], r[c], dx, stay)
                         : kind == kTsDeterministic ? det_timestep(D[c], r[c], dx)
                                                    : cell_timestep(D[c], r[c], dx);
        if (ts == ts) best = min(best, float_key(ts));   // NaN is skipped, as fminf does
    }
    for (int o = 16; o > 0; o >>= 1) best = min(best, __shfl_xor_sync(0xffffffffu, best, o));
    if ((threadIdx.x & 31) == 0) atomicMin(min_key, best);
}

struct DriftParams { float p[8]; };

__global__ void k_diffusivity_drift(int W, int H, int species, int method, DriftParams prm, float L,
                                    float* dx, float* dy, float* rx, float* ry) {
    const int area = W * H;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < area; c += gridDim.x * blockDim.x) {
        const int x = c % W, y = c / W;
        const int64_t i = (int64_t)species * area + c;
        const float px = L / (float)W * ((float)x - (float)W * 0.5f);
        const float py = L / (float)H * ((float)y - (float)H * 0.5f);
        const float* p = prm.p;
        if (method == GPGMP_DRIFT_HOMOGENEOUS) {
            dx[i] = p[0]; dy[i] = p[1]; rx[i] = p[2]; ry[i] = p[3];
        } else if (method == GPGMP_DRIFT_MULTIPLICATIVE_NOISE) {
            const float sx = px + L, sy = py + L;
            dx[i] = (p[0] * p[0]) * (sx * sx) * 0.5f;
            dy[i] = (p[1] * p[1]) * (sy * sy) * 0.5f;
            rx[i] = p[2] * sx;
            ry[i] = p[3] * sy;
        } else if (method == GPGMP_DRIFT_ORNSTEIN_UHLENBECK) {
            dx[i] = p[0]; dy[i] = p[1];
            rx[i] = -(p[2] * px + p[3] * py);
            ry[i] = -(p[4] * px + p[5] * py);
        }
    }
}

// ---- deterministic, reference-compatible ------------------------------------
// Deterministic.cl:17-65 (mirror neighbours), written out of place.
__global__ void k_det_diffuse(const float* __restrict__ in, float* __restrict__ out, int W, int H, int S, int R,
                              const float* __restrict__ D, float dt, float dx2) {
    const int area = W * H;
    const int64_t total = (int64_t)R * S * area;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int c = (int)(i % area);
        const int s = (int)((i / area) % S);
        const int x = c % W, y = c / W;
        const float* p = in + (i - c);
        const float sl = x > 0 ? p[c - 1] : p[c + 1];
        const float sr = x < W - 1 ? p[c + 1] : p[c - 1];
        const float st = y > 0 ? p[c - W] : p[c + W];
        const float sb = y < H - 1 ? p[c + W] : p[c - W];
        const float sh = p[c];
        const float lap = st + sb + sl + sr - 4.0f * sh;
        out[i] = sh + dt * D[s] * lap / dx2;
    }
}

// Deterministic.cl:143-238: 20 classical RK4 substeps per window, clamp at 0.
__global__ void k_rk4(float* state, int S, int area, int R, const gpgmp_reaction* __restrict__ reactions, int nreac,
                      float deltat, const uint32_t* __restrict__ rmask, int rmask_words) {
    extern __shared__ unsigned char smem[];
    gpgmp_reaction* rt = reinterpret_cast<gpgmp_reaction*>(smem);
    float* buf = reinterpret_cast<float*>(smem + sizeof(gpgmp_reaction) * nreac);
    for (int i = threadIdx.x; i < nreac; i += blockDim.x) rt[i] = reactions[i];
    __syncthreads();
    const int64_t total = (int64_t)R * area;
    const int64_t gi = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (gi >= total) return;
    const int r = (int)(gi / area), c = (int)(gi % area);
    const int B = blockDim.x;
    float* x = buf + threadIdx.x;           // [S] stride B
    float* k = buf + (size_t)S * B + threadIdx.x;   // 4 x [S]
    float* y = buf + (size_t)5 * S * B + threadIdx.x;
    float* sp = state + (int64_t)r * S * area + c;
    for (int s = 0; s < S; ++s) x[s * B] = sp[(int64_t)s * area];
    CellReactions on;           // localised reactions contribute nothing where they are off
    on.load(rmask, rmask_words, area, c);
    const int nmax = 20;
    const float h = deltat / (float)nmax;
    for (int it = 0; it < nmax; ++it) {
        for (int stage = 0; stage < 4; ++stage) {
            const float off = stage == 0 ? 0.0f : (stage == 3 ? h : 0.5f * h);
            float* kin = k + (size_t)(stage == 0 ? 0 : stage - 1) * S * B;
            float* kout = k + (size_t)stage * S * B;
            for (int s = 0; s < S; ++s) {
                y[s * B] = stage == 0 ? x[s * B] : x[s * B] + off * kin[s * B];
                kout[s * B] = 0.0f;
            }
            for (int q = 0; q < nreac; ++q) {
                if (!on(q)) continue;
                const gpgmp_reaction& rc = rt[q];
                float law = rc.rate;
                for (int j = 0; j < rc.num_reactants; ++j)
                    for (int m = 0; m < rc.reactant_stoich[j]; ++m) law *= y[rc.reactant_species[j] * B];
                for (int j = 0; j < rc.num_reactants; ++j)
                    kout[rc.reactant_species[j] * B] -= (float)rc.reactant_stoich[j] * law;
                for (int j = 0; j < rc.num_products; ++j)
                    kout[rc.product_species[j] * B] += (float)rc.product_stoich[j] * law;
            }
        }
        for (int s = 0; s < S; ++s) {
            float v = x[s * B] + h / 6.0f * (k[s * B] + 2.0f * k[(S + s) * B] + 2.0f * k[(2 * S + s) * B] +
                                              k[(3 * S + s) * B]);
            x[s * B] = v < 0.0f ? 0.0f : v;
        }
    }
    for (int s = 0; s < S; ++s) sp[(int64_t)s * area] = x[s * B];
}

// Deterministic.cl:71-136 (inhomogeneous drift-diffusion, one direction, one
// species, mirror neighbours): s' = s + dt (D_l s_l + D_r s_r - 2 D s) / dx^2
// - dt (r_r s_r - r_l s_l) / (2 dx), written out of place; the other species'
// planes are copied so that `out` is a whole state.
template <int DIR>
__global__ void k_det_sweep(const float* __restrict__ in, float* __restrict__ out, int W, int H, int S, int R,
                            int species, const float* __restrict__ D, const float* __restrict__ rv, float dt,
                            float dx) {
    const int area = W * H;
    const int64_t total = (int64_t)R * S * area;
    const float dx2 = dx * dx;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int c = (int)(i % area);
        const int s = (int)((i / area) % S);
        if (s != species) {
            out[i] = in[i];
            continue;
        }
        const int x = c % W, y = c / W;
        int lo, hi;
        if (DIR == 0) {
            lo = x > 0 ? c - 1 : c + 1;
            hi = x < W - 1 ? c + 1 : c - 1;
        } else {
            lo = y > 0 ? c - W : c + W;
            hi = y < H - 1 ? c + W : c - W;
        }
        const float* p = in + (i - c);
        const float* Dp = D + (int64_t)species * area;
        const float* rp = rv + (int64_t)species * area;
        const float sl = p[lo] * Dp[lo], sr = p[hi] * Dp[hi], sh = p[c] * Dp[c];
        const float lap = sl + sr - 2.0f * sh;
        const float drift = rp[hi] * p[hi] - rp[lo] * p[lo];
        out[i] = p[c] + dt * lap / dx2 - dt * drift / (2.0f * dx);
    }
}

// ---- alpha-QSS (Mott & Oran 2001), Deterministic.cl:240-522 ------------------------
constexpr int kAqssMaxSpecies = kMaxSpecies;
constexpr int kAqssMaxIter = 100000;    // corrector passes per cell and window before giving up

// production q and destruction d of every species: law = rate * prod x^nu
// (Reaction.cpp:145-162); a reaction adds |net| law to q (net > 0) or d (net < 0)
// of each species whose net stoichiometry it changes (Solver.cpp:961-1004)
__device__ __forceinline__ void aqss_rhs(const gpgmp_reaction* rt, int nreac, int S, const float* y, float* q,
                                         float* d, const CellReactions& on) {
    for (int i = 0; i < S; ++i) { q[i] = 0.0f; d[i] = 0.0f; }
    for (int k = 0; k < nreac; ++k) {
        if (!on(k)) continue;        // localised reaction, off in this cell
        const gpgmp_reaction& rc = rt[k];
        float law = rc.rate;
        for (int j = 0; j < rc.num_reactants; ++j)
            for (int m = 0; m < rc.reactant_stoich[j]; ++m) law *= y[rc.reactant_species[j]];
        // every species of the reaction once, in reactant-then-product order
        for (int pass = 0; pass < 2; ++pass) {
            const int cnt = pass == 0 ? rc.num_reactants : rc.num_products;
            for (int j = 0; j < cnt; ++j) {
                const int sp = pass == 0 ? rc.reactant_species[j] : rc.product_species[j];
                bool seen = false;
                for (int a = 0; a < rc.num_reactants && !seen; ++a)
                    if (rc.reactant_species[a] == sp && (pass == 1 || a < j)) seen = true;
                for (int a = 0; a < rc.num_products && !seen && pass == 1; ++a)
                    if (rc.product_species[a] == sp && a < j) seen = true;
                if (seen) continue;
                int net = 0;
                for (int a = 0; a < rc.num_products; ++a) if (rc.product_species[a] == sp) net += rc.product_stoich[a];
                for (int a = 0; a < rc.num_reactants; ++a) if (rc.reactant_species[a] == sp) net -= rc.reactant_stoich[a];
                if (net > 0) q[sp] += (float)net * law;
                else if (net < 0) d[sp] += (float)(-net) * law;
            }
        }
    }
}

__device__ __forceinline__ float aqss_alpha(float r) {
    return (180.0f + r * (60.0f + r * (11.0f + r))) / (360.0f + r * (60.0f + r * (12.0f + r)));
}

// One window of length dtg for the species x[0..S) of one cell.  A retried step
// restarts its predictor from the saved start state with the reduced step size
// (Mott & Oran's method).  literal: the reference's form instead -- the predictor
// takes the current production/destruction and the outer step's size
// (Deterministic.cl:381-387, which never shrinks on a retry, so a species growing
// from zero can be rejected forever) and the corrector coefficient as printed
// (`180.*+rtaub`, :424).  Returns GPGMP_SIM_EVENT_CAP if the step control did not
// finish within kAqssMaxIter passes.
__device__ int aqss_cell(const gpgmp_reaction* rt, int nreac, int S, float* y, float dtg, bool literal,
                         const CellReactions& on) {
    const float epsmin = 1e-2f, sqreps = 0.5f, epscl = 100.0f, epsmax = 10.0f, tfd = 1.000008f, dtmin = 1e-15f,
                ymin = 1e-20f;
    constexpr int itermax = 2;
    float q[kAqssMaxSpecies], d[kAqssMaxSpecies], ys[kAqssMaxSpecies], qs[kAqssMaxSpecies], ds[kAqssMaxSpecies],
        rtaus[kAqssMaxSpecies], scr[kAqssMaxSpecies], y1[kAqssMaxSpecies];
    float tn = 0.0f;
    for (int i = 0; i < S; ++i) y[i] = fmaxf(y[i], ymin);
    aqss_rhs(rt, nreac, S, y, q, d, on);
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
        const float ts = tn;
        const float dtcurrent = dt;
        for (int i = 0; i < S; ++i) {
            ys[i] = y[i];
            qs[i] = q[i];
            ds[i] = d[i];
            rtaus[i] = dtcurrent * d[i] / y[i];
        }
        while (dtg > tn * tfd) {
            if (++passes > kAqssMaxIter) return GPGMP_SIM_EVENT_CAP;
            for (int i = 0; i < S; ++i) {
                if (literal) {
                    const float rtaui = dtcurrent * d[i] / y[i];
                    scr[i] = (q[i] - d[i]) / (1.0f + aqss_alpha(rtaui) * rtaui);
                } else {
                    const float rtaui = dt * ds[i] / ys[i];
                    scr[i] = (qs[i] - ds[i]) / (1.0f + aqss_alpha(rtaui) * rtaui);
                }
            }
            float eps = 1e-10f;
            for (int iteration = 0; iteration < itermax; ++iteration) {
                for (int i = 0; i < S; ++i) y[i] = fmaxf(ys[i] + dt * scr[i], ymin);
                if (iteration == 0) {
                    tn = ts + dt;
                    for (int i = 0; i < S; ++i) y1[i] = y[i];
                }
                aqss_rhs(rt, nreac, S, y, q, d, on);
                eps = 1e-10f;
                for (int i = 0; i < S; ++i) {
                    const float rtaub = 0.5f * (rtaus[i] + dt * d[i] / y[i]);
                    const float alpha =
                        literal ? (180.0f * rtaub * (60.0f + rtaub * (11.0f + rtaub))) /
                                      (360.0f + rtaub * (60.0f + rtaub * (12.0f + rtaub)))
                                : aqss_alpha(rtaub);
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
            if (dt <= dtmin + 1e-16f * tn) {
                dt = dtg - ts;
                dt = fminf(dtmin, fabsf(dt));
            }
            const float stab = 0.01f;     // the stability test needs itermax >= 3
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
        aqss_rhs(rt, nreac, S, y, q, d, on);
    }
    return 0;
}

__global__ void k_aqss(float* state, int S, int area, int R, const gpgmp_reaction* __restrict__ reactions, int nreac,
                       float deltat, int literal, int32_t* status, const uint32_t* __restrict__ rmask,
                       int rmask_words) {
    extern __shared__ unsigned char smem[];
    gpgmp_reaction* rt = reinterpret_cast<gpgmp_reaction*>(smem);
    for (int i = threadIdx.x; i < nreac; i += blockDim.x) rt[i] = reactions[i];
    __syncthreads();
    const int64_t total = (int64_t)R * area;
    for (int64_t gi = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; gi < total;
         gi += (int64_t)gridDim.x * blockDim.x) {
        const int r = (int)(gi / area), c = (int)(gi % area);
        float* sp = state + (int64_t)r * S * area + c;
        float y[kAqssMaxSpecies];
        for (int s = 0; s < S; ++s) y[s] = sp[(int64_t)s * area];
        CellReactions on;
        on.load(rmask, rmask_words, area, c);
        const int e = aqss_cell(rt, nreac, S, y, deltat, literal != 0, on);
        for (int s = 0; s < S; ++s) sp[(int64_t)s * area] = y[s];
        if (e) atomicOr(&status[r], e);
    }
}

inline unsigned grid_for(int64_t n, int threads) {
    int64_t b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > 148 * 64) b = 148 * 64;
    return (unsigned)b;
}

}  // namespace

cudaError_t launch_init_poisson(const GridDesc& g, Planes planes, uint32_t seed, const float* d_lambda,
                                cudaStream_t st) {
    const int area = g.W * g.H;
    k_init_poisson<<<grid_for((int64_t)g.R * area, 256), 256, 0, st>>>(planes, g.S, area, g.R, seed, d_lambda);
    return cudaGetLastError();
}

namespace {
template <bool MASKED, int NTH>
cudaError_t launch_ssa_t(const GridDesc& g, Planes planes, const gpgmp_reaction* d_reactions, int nreac,
                         uint32_t seed, uint32_t step_seed, float window, int32_t* d_status, cudaStream_t st) {
    const int area = g.W * g.H;
    const int64_t total = (int64_t)g.R * area;
    const size_t smem = sizeof(gpgmp_reaction) * nreac + sizeof(uint32_t) * 4 * nreac +
                        sizeof(float) * (size_t)nreac * NTH + sizeof(int) * g.S * NTH;
    const unsigned blocks = (unsigned)((total + NTH - 1) / NTH);
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(k_ssa<MASKED, NTH>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    k_ssa<MASKED, NTH><<<blocks, NTH, smem, st>>>(planes, g.S, area, g.R, d_reactions, nreac, seed, step_seed, window,
                                                  d_status, g.rmask, g.rmask_words);
    return cudaGetLastError();
}
template <bool MASKED>
cudaError_t launch_ssa_m(const GridDesc& g, Planes planes, const gpgmp_reaction* d_reactions, int nreac,
                         uint32_t seed, uint32_t step_seed, float window, int32_t* d_status, cudaStream_t st) {
    switch (kSsaThreadChoices[g.ssa_threads]) {
        case 64: return launch_ssa_t<MASKED, 64>(g, planes, d_reactions, nreac, seed, step_seed, window, d_status, st);
        case 256: return launch_ssa_t<MASKED, 256>(g, planes, d_reactions, nreac, seed, step_seed, window, d_status, st);
        default: return launch_ssa_t<MASKED, 128>(g, planes, d_reactions, nreac, seed, step_seed, window, d_status, st);
    }
}

template <int MODE, int TW, int TH>
cudaError_t launch_tile_t(const GridDesc& g, const int32_t* in, int32_t* out, int species, uint32_t seed,
                          uint32_t step_seed, float pmove, const float* d_D, const float* d_r, float dt, float dx,
                          int fpe, cudaStream_t st) {
    dim3 grid((g.W + TW - 1) / TW, (g.H + TH - 1) / TH, g.R);
    const int4 bm = make_int4(g.bmask[0], g.bmask[1], g.bmask[2], g.bmask[3]);
    k_diffuse_tile<MODE, TW, TH><<<grid, NT, 0, st>>>(in, out, g.W, g.H, g.S, species, seed, step_seed, pmove, bm,
                                                      d_D, d_r, dt, dx, fpe);
    return cudaGetLastError();
}
template <int MODE>
cudaError_t launch_tile(const GridDesc& g, const int32_t* in, int32_t* out, int species, uint32_t seed,
                        uint32_t step_seed, float pmove, const float* d_D, const float* d_r, float dt, float dx,
                        int fpe, cudaStream_t st) {
#define GPGMP_TILE(I)                                                                                              \
    case I:                                                                                                        \
        return launch_tile_t<MODE, kTileW[I], kTileH[I]>(g, in, out, species, seed, step_seed, pmove, d_D, d_r, dt, \
                                                          dx, fpe, st);
    switch (g.tile) {
        GPGMP_TILE(1)
        GPGMP_TILE(2)
        GPGMP_TILE(3)
        GPGMP_TILE(4)
        GPGMP_TILE(5)
        default: GPGMP_TILE(0)
    }
#undef GPGMP_TILE
}
}  // namespace

void diffusion_tile_shape(int index, int* w, int* h) {
    *w = kTileW[index];
    *h = kTileH[index];
}
int ssa_thread_choice(int index) { return kSsaThreadChoices[index]; }

cudaError_t launch_ssa(const GridDesc& g, Planes planes, const gpgmp_reaction* d_reactions, int nreac,
                       uint32_t seed, uint32_t step_seed, float window, int32_t* d_status, cudaStream_t st) {
    if (nreac <= 0) return cudaSuccess;
    return g.rmask ? launch_ssa_m<true>(g, planes, d_reactions, nreac, seed, step_seed, window, d_status, st)
                   : launch_ssa_m<false>(g, planes, d_reactions, nreac, seed, step_seed, window, d_status, st);
}

cudaError_t launch_homog_diffuse(const GridDesc& g, const int32_t* in, int32_t* out, int species, uint32_t seed,
                                 uint32_t step_seed, float pmove, cudaStream_t st) {
    return launch_tile<0>(g, in, out, species, seed, step_seed, pmove, nullptr, nullptr, 0.f, 0.f, 0, st);
}

cudaError_t launch_source(const GridDesc& g, int32_t* plane_base, int species, uint32_t seed, uint32_t step_seed,
                          int boundary, int count, float pi, cudaStream_t st) {
    k_source<<<grid_for((int64_t)g.R * g.W, 128), 128, 0, st>>>(plane_base, g.W, g.H, g.S, g.R, species, seed,
                                                                 step_seed, boundary, count, pi);
    return cudaGetLastError();
}

cudaError_t launch_sweep(const GridDesc& g, const int32_t* in, int32_t* out, int species, int sweep_y,
                         uint32_t seed, uint32_t step_seed, const float* d_D, const float* d_r, float dt, float dx,
                         cudaStream_t st, int fpe) {
    return sweep_y ? launch_tile<2>(g, in, out, species, seed, step_seed, 0.f, d_D, d_r, dt, dx, fpe, st)
                   : launch_tile<1>(g, in, out, species, seed, step_seed, 0.f, d_D, d_r, dt, dx, fpe, st);
}

cudaError_t launch_det_sweep(const GridDesc& g, const float* in, float* out, int species, int sweep_y,
                             const float* d_D, const float* d_r, float dt, float dx, cudaStream_t st) {
    const int64_t total = (int64_t)g.R * g.S * g.W * g.H;
    if (!sweep_y)
        k_det_sweep<0><<<grid_for(total, 256), 256, 0, st>>>(in, out, g.W, g.H, g.S, g.R, species, d_D, d_r, dt, dx);
    else
        k_det_sweep<1><<<grid_for(total, 256), 256, 0, st>>>(in, out, g.W, g.H, g.S, g.R, species, d_D, d_r, dt, dx);
    return cudaGetLastError();
}

cudaError_t launch_aqss(const GridDesc& g, float* state, const gpgmp_reaction* d_reactions, int nreac, float deltat,
                        int literal, int32_t* d_status, cudaStream_t st) {
    if (nreac <= 0) return cudaSuccess;
    const int area = g.W * g.H;
    const int64_t total = (int64_t)g.R * area;
    const int threads = 128;
    const size_t smem = sizeof(gpgmp_reaction) * nreac;
    k_aqss<<<grid_for(total, threads), threads, smem, st>>>(state, g.S, area, g.R, d_reactions, nreac, deltat, literal,
                                                             d_status, g.rmask, g.rmask_words);
    return cudaGetLastError();
}

cudaError_t launch_timestep(int area, const float* d_D, const float* d_r, float dx, uint32_t* d_min_key,
                            cudaStream_t st, int kind, float stay) {
    cudaError_t e = cudaMemsetAsync(d_min_key, 0xff, sizeof(uint32_t), st);
    if (e != cudaSuccess) return e;
    k_timestep<<<grid_for(area, 256), 256, 0, st>>>(area, d_D, d_r, dx, d_min_key, kind, stay);
    return cudaGetLastError();
}

// inhomogeneous_computeMomentsX + reduceMomentsBlocks (StochasticInhomogeneousDriftDiffusion.cl:5-84)
// and getMeanX (helpers.cl:18-21): MeanX = L / W * (sum x n / sum n - W / 2) of one
// species plane, the sums taken exactly in 64-bit integers.
__global__ void k_moments_sum(const int32_t* __restrict__ plane, int W, int area, unsigned long long* sums) {
    unsigned long long mx = 0, n = 0;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < area; c += gridDim.x * blockDim.x) {
        const long long v = plane[c] > 0 ? plane[c] : 0;
        mx += (unsigned long long)(v * (c % W));
        n += (unsigned long long)v;
    }
    for (int o = 16; o > 0; o >>= 1) {
        mx += __shfl_xor_sync(0xffffffffu, mx, o);
        n += __shfl_xor_sync(0xffffffffu, n, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&sums[0], mx);
        atomicAdd(&sums[1], n);
    }
}
__global__ void k_moments_finish(const unsigned long long* sums, int W, float L, float* meanx) {
    const float tmp = (float)sums[0] / (float)sums[1];
    *meanx = L / (float)W * (tmp - (float)W / 2.0f);
}

cudaError_t launch_moments(const int32_t* plane, int W, int H, float L, unsigned long long* d_sums, float* d_meanx,
                           cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(d_sums, 0, 2 * sizeof(unsigned long long), st);
    if (e != cudaSuccess) return e;
    const int area = W * H;
    k_moments_sum<<<grid_for(area, 256), 256, 0, st>>>(plane, W, area, d_sums);
    k_moments_finish<<<1, 1, 0, st>>>(d_sums, W, L, d_meanx);
    return cudaGetLastError();
}

cudaError_t launch_diffusivity_drift(const GridDesc& g, int species, int method, const float* params, float L,
                                     float* dx, float* dy, float* rx, float* ry, cudaStream_t st) {
    DriftParams p;
    for (int i = 0; i < 8; ++i) p.p[i] = params[i];
    k_diffusivity_drift<<<grid_for((int64_t)g.W * g.H, 256), 256, 0, st>>>(g.W, g.H, species, method, p, L, dx, dy,
                                                                            rx, ry);
    return cudaGetLastError();
}

cudaError_t launch_det_diffuse(const GridDesc& g, const float* in, float* out, const float* d_D, float dt,
                               float dx2, cudaStream_t st) {
    const int64_t total = (int64_t)g.R * g.S * g.W * g.H;
    k_det_diffuse<<<grid_for(total, 256), 256, 0, st>>>(in, out, g.W, g.H, g.S, g.R, d_D, dt, dx2);
    return cudaGetLastError();
}

cudaError_t launch_rk4(const GridDesc& g, float* state, const gpgmp_reaction* d_reactions, int nreac, float deltat,
                       cudaStream_t st) {
    if (nreac <= 0) return cudaSuccess;
    const int threads = 64;
    const int area = g.W * g.H;
    const int64_t total = (int64_t)g.R * area;
    const size_t smem = sizeof(gpgmp_reaction) * nreac + sizeof(float) * 6 * g.S * threads;
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(k_rk4, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    k_rk4<<<(unsigned)((total + threads - 1) / threads), threads, smem, st>>>(state, g.S, area, g.R, d_reactions,
                                                                             nreac, deltat, g.rmask, g.rmask_words);
    return cudaGetLastError();
}

}  // namespace gpgmp
