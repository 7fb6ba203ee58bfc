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

constexpr int kSsaThreads = 128;
constexpr int kIncMinReactions = 6;   // networks above this size keep per-reaction hazards
constexpr int TW = 32, TH = 16, NT = 256;

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

__global__ void __launch_bounds__(kSsaThreads) k_ssa(Planes planes, int S, int area, int R,
                                                     const gpgmp_reaction* __restrict__ reactions, int nreac,
                                                     uint32_t seed, uint32_t step_seed, float window,
                                                     int32_t* __restrict__ status) {
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
    const int e = nreac > kIncMinReactions ? ssa_cell_inc(rt, deps, nreac, x, kSsaThreads, hs + threadIdx.x, st, window)
                                           : ssa_cell(rt, nreac, x, kSsaThreads, st, window);
    for (int s = 0; s < S; ++s) planes.p[s][((int64_t)r * S + s) * area + c] = x[s * kSsaThreads];
    if (e) atomicOr(&status[r], e);
}

// MODE 0: 2-D homogeneous jumps; 1: drift-diffusion sweep in x; 2: sweep in y.
// A block owns a TW x TH tile, samples the lost counts of the tile and of its
// one-cell halo (recomputed, the streams are keyed by cell) into shared memory,
// then gathers.  Reads `in`, writes `out`: no block reads what another writes.
template <int MODE>
__global__ void __launch_bounds__(NT) k_diffuse_tile(const int* __restrict__ in, int* __restrict__ out, int W, int H,
                                                     int S, int species, uint32_t seed, uint32_t step_seed,
                                                     float pmove, int4 bm4, const float* __restrict__ Df,
                                                     const float* __restrict__ rf, float dt, float dx) {
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
                sweep_lost(n, Df[fi], rf[fi], dt, dx, st, gx == 0, gx == W - 1, bm[0], bm[1], &l[0], &l[1]);
            } else {
                const int64_t fi = (int64_t)species * area + c;
                sweep_lost(n, Df[fi], rf[fi], dt, dx, st, gy == 0, gy == H - 1, bm[2], bm[3], &l[0], &l[1]);
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
                           uint32_t* min_key) {
    uint32_t best = 0xffffffffu;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < area; c += gridDim.x * blockDim.x)
    {
        const float ts = cell_timestep(D[c], r[c], dx);
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
                      float deltat) {
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

cudaError_t launch_ssa(const GridDesc& g, Planes planes, const gpgmp_reaction* d_reactions, int nreac,
                       uint32_t seed, uint32_t step_seed, float window, int32_t* d_status, cudaStream_t st) {
    if (nreac <= 0) return cudaSuccess;
    const int area = g.W * g.H;
    const int64_t total = (int64_t)g.R * area;
    const size_t smem = sizeof(gpgmp_reaction) * nreac + sizeof(uint32_t) * 4 * nreac +
                        sizeof(float) * (size_t)nreac * kSsaThreads + sizeof(int) * g.S * kSsaThreads;
    const unsigned blocks = (unsigned)((total + kSsaThreads - 1) / kSsaThreads);
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(k_ssa, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    k_ssa<<<blocks, kSsaThreads, smem, st>>>(planes, g.S, area, g.R, d_reactions, nreac, seed, step_seed, window,
                                              d_status);
    return cudaGetLastError();
}

cudaError_t launch_homog_diffuse(const GridDesc& g, const int32_t* in, int32_t* out, int species, uint32_t seed,
                                 uint32_t step_seed, float pmove, cudaStream_t st) {
    dim3 grid((g.W + TW - 1) / TW, (g.H + TH - 1) / TH, g.R);
    int4 bm = make_int4(g.bmask[0], g.bmask[1], g.bmask[2], g.bmask[3]);
    k_diffuse_tile<0><<<grid, NT, 0, st>>>(in, out, g.W, g.H, g.S, species, seed, step_seed, pmove, bm, nullptr,
                                            nullptr, 0.f, 0.f);
    return cudaGetLastError();
}

cudaError_t launch_source(const GridDesc& g, int32_t* plane_base, int species, uint32_t seed, uint32_t step_seed,
                          int boundary, int count, float pi, cudaStream_t st) {
    k_source<<<grid_for((int64_t)g.R * g.W, 128), 128, 0, st>>>(plane_base, g.W, g.H, g.S, g.R, species, seed,
                                                                 step_seed, boundary, count, pi);
    return cudaGetLastError();
}

cudaError_t launch_sweep(const GridDesc& g, const int32_t* in, int32_t* out, int species, int sweep_y,
                         uint32_t seed, uint32_t step_seed, const float* d_D, const float* d_r, float dt, float dx,
                         cudaStream_t st) {
    dim3 grid((g.W + TW - 1) / TW, (g.H + TH - 1) / TH, g.R);
    int4 bm = make_int4(g.bmask[0], g.bmask[1], g.bmask[2], g.bmask[3]);
    if (!sweep_y)
        k_diffuse_tile<1><<<grid, NT, 0, st>>>(in, out, g.W, g.H, g.S, species, seed, step_seed, 0.f, bm, d_D, d_r,
                                                dt, dx);
    else
        k_diffuse_tile<2><<<grid, NT, 0, st>>>(in, out, g.W, g.H, g.S, species, seed, step_seed, 0.f, bm, d_D, d_r,
                                                dt, dx);
    return cudaGetLastError();
}

cudaError_t launch_timestep(int area, const float* d_D, const float* d_r, float dx, uint32_t* d_min_key,
                            cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(d_min_key, 0xff, sizeof(uint32_t), st);
    if (e != cudaSuccess) return e;
    k_timestep<<<grid_for(area, 256), 256, 0, st>>>(area, d_D, d_r, dx, d_min_key);
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
                                                                             nreac, deltat);
    return cudaGetLastError();
}

}  // namespace gpgmp
