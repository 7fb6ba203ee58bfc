// Deterministic reaction-diffusion (Gray-Scott kinetics) and its adjoint.
//
// Model: the reference's Gray-Scott network (exec/src/tests/GrayScottModel.cpp:14-60;
// U+2V->3V, U->0 at F, V->0 at F+k, 0->U at F, with the deterministic laws of
// Reaction.cpp:145-162) on a periodic N x N lattice (h = 1), explicit Euler steps,
// 5-point Laplacian and an optional constant drift (vx, vy) by central differences
// (the drift stencil of Deterministic.cl:71-136 with constant velocity):
//   u' = u + dt (Du lap u - vx dx u - vy dy u - u v^2 + F (1 - u))
//   v' = v + dt (Dv lap v - vx dx v - vy dy v + u v^2 - (F + k) v)
//
// B200 design: the whole lattice lives in the shared memory of ONE thread-block
// cluster (CL CTAs, N/CL rows each, double-buffered, one halo row above and
// below).  A step is: cluster barrier, copy the two halo rows from the
// neighbouring CTAs' shared memory (DSMEM), block barrier, update the own rows.
// No global-memory traffic inside the time loop except the optional per-step
// state stream the adjoint's recomputation needs.
//
// The adjoint runs the transposed step backwards over a segment of stored states,
// with the adjoint fields in cluster shared memory the same way, and accumulates
// the parameter gradients (F, k, Du, Dv, vx, vy) in double per thread.
#include <cooperative_groups.h>
#include <cstdint>
#include <cstdio>
#include <mutex>
#include <type_traits>
#include <vector>
#include <cuda_runtime.h>
#include "gs_kernels.h"
#include "host_common.h"

namespace cg = cooperative_groups;

namespace gpgmp {
namespace {

constexpr int kThreads = 512;

template <typename T>
struct GSArgs {
    int n, steps;
    T F, k, Du, Dv, vx, vy, dt;
};

// shared layout: [buf 0/1][field u/v][rows + 2][n]
template <typename T>
__device__ __forceinline__ T* plane(T* sm, int buf, int field, int rp, int n) {
    return sm + ((size_t)(buf * 2 + field) * (rp + 2)) * n;
}

template <typename T>
__device__ __forceinline__ void fill_halo(cg::cluster_group& cl, T* sm, int buf, int rp, int n) {
    const unsigned rank = cl.block_rank();
    const unsigned nb = cl.num_blocks();
    const unsigned up = (rank + nb - 1) % nb, down = (rank + 1) % nb;
    for (int f = 0; f < 2; ++f) {
        T* p = plane(sm, buf, f, rp, n);
        const T* pu = cl.map_shared_rank(p, up);
        const T* pd = cl.map_shared_rank(p, down);
        for (int c = threadIdx.x; c < n; c += blockDim.x) {
            p[c] = pu[(size_t)rp * n + c];                 // row 0 <- upper neighbour's last own row
            p[(size_t)(rp + 1) * n + c] = pd[(size_t)n + c];  // row rp+1 <- lower neighbour's first own row
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(kThreads, 1) k_gs_forward(GSArgs<T> a, const T* __restrict__ u0,
                                                           const T* __restrict__ v0, T* __restrict__ uo,
                                                           T* __restrict__ vo, T* __restrict__ trace,
                                                           int trace_every) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* sm = reinterpret_cast<T*>(smem_raw);
    cg::cluster_group cl = cg::this_cluster();
    const int n = a.n;
    const int rp = n / (int)cl.num_blocks();
    const int r0 = (int)cl.block_rank() * rp;
    const size_t nn = (size_t)n * n;
    for (int i = threadIdx.x; i < rp * n; i += blockDim.x) {
        plane(sm, 0, 0, rp, n)[n + i] = u0[(size_t)r0 * n + i];
        plane(sm, 0, 1, rp, n)[n + i] = v0[(size_t)r0 * n + i];
    }
    const T one = T(1), half = T(0.5), four = T(4);
    const T Fk = a.F + a.k;
    for (int s = 0; s < a.steps; ++s) {
        const int cur = s & 1, nxt = cur ^ 1;
        cl.sync();
        fill_halo(cl, sm, cur, rp, n);
        if (trace && s % trace_every == 0) {
            T* dst = trace + (size_t)(2 * (s / trace_every)) * nn + (size_t)r0 * n;
            for (int i = threadIdx.x; i < rp * n; i += blockDim.x) {
                dst[i] = plane(sm, cur, 0, rp, n)[n + i];
                dst[nn + i] = plane(sm, cur, 1, rp, n)[n + i];
            }
        }
        __syncthreads();
        const T* U = plane(sm, cur, 0, rp, n);
        const T* V = plane(sm, cur, 1, rp, n);
        T* Un = plane(sm, nxt, 0, rp, n);
        T* Vn = plane(sm, nxt, 1, rp, n);
        for (int i = threadIdx.x; i < rp * n; i += blockDim.x) {
            const int r = i / n + 1, c = i % n;
            const int cl_ = c == 0 ? n - 1 : c - 1, cr = c == n - 1 ? 0 : c + 1;
            const size_t o = (size_t)r * n;
            const T uc = U[o + c], vc = V[o + c];
            const T uL = U[o + cl_], uR = U[o + cr], uU = U[o - n + c], uD = U[o + n + c];
            const T vL = V[o + cl_], vR = V[o + cr], vU = V[o - n + c], vD = V[o + n + c];
            const T lu = uL + uR + uU + uD - four * uc;
            const T lv = vL + vR + vU + vD - four * vc;
            const T uvv = uc * vc * vc;
            const T adv_u = a.vx * (uR - uL) * half + a.vy * (uD - uU) * half;
            const T adv_v = a.vx * (vR - vL) * half + a.vy * (vD - vU) * half;
            const T un = uc + a.dt * (a.Du * lu - adv_u - uvv + a.F * (one - uc));
            const T vn = vc + a.dt * (a.Dv * lv - adv_v + uvv - Fk * vc);
            Un[o + c] = un;
            Vn[o + c] = vn;
        }
    }
    __syncthreads();
    const int fin = a.steps & 1;
    for (int i = threadIdx.x; i < rp * n; i += blockDim.x) {
        uo[(size_t)r0 * n + i] = plane(sm, fin, 0, rp, n)[n + i];
        vo[(size_t)r0 * n + i] = plane(sm, fin, 1, rp, n)[n + i];
    }
    cl.sync();  // no CTA may exit while a neighbour can still read its shared memory
}

// Adjoint over one segment: states[j] (j = 0..len-1, each [u | v] of n*n) are the
// forward states before step j of the segment; lam enters as the adjoint after the
// segment and leaves as the adjoint at its start.
template <typename T>
__global__ void __launch_bounds__(kThreads, 1) k_gs_adjoint(GSArgs<T> a, const T* __restrict__ states, int len,
                                                           const T* __restrict__ lu_in, const T* __restrict__ lv_in,
                                                           T* __restrict__ lu_out, T* __restrict__ lv_out,
                                                           double* __restrict__ grad, int* __restrict__ err) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* sm = reinterpret_cast<T*>(smem_raw);
    __shared__ double red[6][kThreads / 32];
    cg::cluster_group cl = cg::this_cluster();
    const int n = a.n;
    const int rp = n / (int)cl.num_blocks();
    const int r0 = (int)cl.block_rank() * rp;
    const size_t nn = (size_t)n * n;
    for (int i = threadIdx.x; i < rp * n; i += blockDim.x) {
        plane(sm, 0, 0, rp, n)[n + i] = lu_in[(size_t)r0 * n + i];
        plane(sm, 0, 1, rp, n)[n + i] = lv_in[(size_t)r0 * n + i];
    }
    double gF = 0, gk = 0, gDu = 0, gDv = 0, gvx = 0, gvy = 0;
    const T one = T(1), two = T(2), half = T(0.5), four = T(4);
    const T Fk = a.F + a.k;
    for (int j = len - 1, s = 0; j >= 0; --j, ++s) {
        const int cur = s & 1, nxt = cur ^ 1;
        cl.sync();
        fill_halo(cl, sm, cur, rp, n);
        __syncthreads();
        const T* A = plane(sm, cur, 0, rp, n);
        const T* B = plane(sm, cur, 1, rp, n);
        T* An = plane(sm, nxt, 0, rp, n);
        T* Bn = plane(sm, nxt, 1, rp, n);
        const T* Us = states + (size_t)(2 * j) * nn;
        const T* Vs = Us + nn;
        for (int i = threadIdx.x; i < rp * n; i += blockDim.x) {
            const int r = i / n + 1, c = i % n;
            const int cl_ = c == 0 ? n - 1 : c - 1, cr = c == n - 1 ? 0 : c + 1;
            const size_t o = (size_t)r * n;
            const int gr = r0 + r - 1;
            const int gu = gr == 0 ? n - 1 : gr - 1, gd = gr == n - 1 ? 0 : gr + 1;
            const T uc = Us[(size_t)gr * n + c], vc = Vs[(size_t)gr * n + c];
            const T uL = Us[(size_t)gr * n + cl_], uR = Us[(size_t)gr * n + cr];
            const T uU = Us[(size_t)gu * n + c], uD = Us[(size_t)gd * n + c];
            const T vL = Vs[(size_t)gr * n + cl_], vR = Vs[(size_t)gr * n + cr];
            const T vU = Vs[(size_t)gu * n + c], vD = Vs[(size_t)gd * n + c];
            const T ac = A[o + c], bc = B[o + c];
            const T aL = A[o + cl_], aR = A[o + cr], aU = A[o - n + c], aD = A[o + n + c];
            const T bL = B[o + cl_], bR = B[o + cr], bU = B[o - n + c], bD = B[o + n + c];
            const T lap_a = aL + aR + aU + aD - four * ac;
            const T lap_b = bL + bR + bU + bD - four * bc;
            const T dxa = (aR - aL) * half, dya = (aD - aU) * half;
            const T dxb = (bR - bL) * half, dyb = (bD - bU) * half;
            const T v2 = vc * vc, uv = uc * vc;
            An[o + c] = ac + a.dt * (a.Du * lap_a + a.vx * dxa + a.vy * dya + ac * (-v2 - a.F) + bc * v2);
            Bn[o + c] = bc + a.dt * (a.Dv * lap_b + a.vx * dxb + a.vy * dyb + ac * (-two * uv) + bc * (two * uv - Fk));
            const double lu = (double)(uL + uR + uU + uD - four * uc);
            const double lv = (double)(vL + vR + vU + vD - four * vc);
            gF += (double)ac * (1.0 - (double)uc) - (double)bc * (double)vc;
            gk += -(double)bc * (double)vc;
            gDu += (double)ac * lu;
            gDv += (double)bc * lv;
            gvx += -(double)ac * (double)((uR - uL) * half) - (double)bc * (double)((vR - vL) * half);
            gvy += -(double)ac * (double)((uD - uU) * half) - (double)bc * (double)((vD - vU) * half);
        }
    }
    __syncthreads();
    const int fin = len & 1;
    for (int i = threadIdx.x; i < rp * n; i += blockDim.x) {
        lu_out[(size_t)r0 * n + i] = plane(sm, fin, 0, rp, n)[n + i];
        lv_out[(size_t)r0 * n + i] = plane(sm, fin, 1, rp, n)[n + i];
    }
    double g[6] = {gF, gk, gDu, gDv, gvx, gvy};
    const double dtd = (double)a.dt;
#pragma unroll
    for (int q = 0; q < 6; ++q) {
        double v = g[q] * dtd;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0) red[q][threadIdx.x >> 5] = v;
    }
    __syncthreads();
    if (threadIdx.x < 6) {
        double v = 0;
        for (int w = 0; w < kThreads / 32; ++w) v += red[threadIdx.x][w];
        atomicAdd(&grad[threadIdx.x], v);
    }
    cl.sync();
}


// ---- fast path: column walk with a split-phase cluster barrier -------------------
// Block (BX, BY): thread (tx, ty) owns columns tx, tx + BX, ... and the RPT rows
// 1 + ty RPT .. (ty + 1) RPT of its CTA's slab; walking down a column it keeps the
// rows above, at and below the cell in registers (three shared loads per cell and
// field).  Per step: the interior rows (2 .. rp-1, which need no halo) are updated
// while the cluster barrier of the previous step completes; after the wait the
// two edge rows are updated reading the neighbouring slabs' edge rows directly from
// their shared memory (DSMEM); then a block barrier and the arrive for this step.
// A CTA's edge rows of a buffer are rewritten only after the next wait, which
// needs every neighbour's arrive, which follows its reads: no read-after-write or
// write-after-read race across CTAs.
__device__ __forceinline__ void cluster_arrive() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void cluster_wait() {
    asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}
// Arrive without a fence of its own: threads that wrote data other CTAs will read
// (the edge rows) release it with cluster_release() first; the rest only signal.
__device__ __forceinline__ void cluster_arrive_relaxed() {
    asm volatile("barrier.cluster.arrive.relaxed.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void cluster_release() { asm volatile("fence.acq_rel.cluster;\n" ::: "memory"); }

// Folded constants of one explicit step, applied in increment form (the small
// update is formed first and added to the cell's value, which keeps float32
// rounding at the size of the update):
//   u' = u + du lap u + hx (uL - uR) + hy (uU - uD) + dtF (1 - u) - dt u v^2
//   v' = v + dv lap v + hx (vL - vR) + hy (vU - vD) - dtFk v     + dt u v^2
// with du = dt Du, dv = dt Dv, hx = dt vx / 2, hy = dt vy / 2, dtF = dt F,
// dtFk = dt (F + k).
template <typename T>
struct GSCoef {
    T du, dv, hx, hy, dt, dtF, dtFk;
    bool drift;
    __device__ __forceinline__ explicit GSCoef(const GSArgs<T>& a) {
        du = a.dt * a.Du;
        dv = a.dt * a.Dv;
        hx = a.dt * a.vx * T(0.5);
        hy = a.dt * a.vy * T(0.5);
        dt = a.dt;
        dtF = a.dt * a.F;
        dtFk = a.dt * (a.F + a.k);
        drift = a.vx != T(0) || a.vy != T(0);
    }
};

template <typename T>
__device__ __forceinline__ void gs_update(const GSCoef<T>& k, T uU, T uC, T uD, T uL, T uR, T vU, T vC, T vD, T vL,
                                          T vR, T* un, T* vn) {
    const T uvv = uC * vC * vC;
    const T lu = fma(T(-4), uC, (uL + uR) + (uU + uD));
    const T lv = fma(T(-4), vC, (vL + vR) + (vU + vD));
    T a = fma(k.du, lu, fma(-k.dtF, uC, k.dtF));
    T b = fma(-k.dtFk, vC, k.dv * lv);
    if (k.drift) {
        a = fma(k.hx, uL - uR, fma(k.hy, uU - uD, a));
        b = fma(k.hx, vL - vR, fma(k.hy, vU - vD, b));
    }
    *un = uC + fma(-k.dt, uvv, a);
    *vn = vC + fma(k.dt, uvv, b);
}

// Forward kernel with the lattice side N known at compile time.
template <typename T, int N>
__global__ void __launch_bounds__(1024, 1) k_gs_forward_cw(GSArgs<T> a, const T* __restrict__ u0,
                                                          const T* __restrict__ v0, T* __restrict__ uo,
                                                          T* __restrict__ vo, T* __restrict__ trace,
                                                          int trace_every) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* sm = reinterpret_cast<T*>(smem_raw);
    cg::cluster_group cl = cg::this_cluster();
    const int rp = N / (int)cl.num_blocks();
    const int r0 = (int)cl.block_rank() * rp;
    constexpr int NN = N * N;
    const int BX = blockDim.x, BY = blockDim.y;
    const int tid = threadIdx.y * BX + threadIdx.x;
    const int nthr = BX * BY;
    const int rpt = rp / BY;
    const int rb = 1 + threadIdx.y * rpt;
    const int ilo = rb < 2 ? 2 : rb;
    const int ihi = rb + rpt - 1 > rp - 1 ? rp - 1 : rb + rpt - 1;
    const unsigned rank = cl.block_rank(), nb = cl.num_blocks();
    const unsigned up = (rank + nb - 1) % nb, down = (rank + 1) % nb;
    const GSCoef<T> k(a);
    const int PL = (rp + 2) * N;                // one plane: [rp + 2][N]; layout [buf][field]
    for (int i = tid; i < rp * N; i += nthr) {
        sm[N + i] = u0[r0 * N + i];
        sm[PL + N + i] = v0[r0 * N + i];
    }
    __syncthreads();
    cluster_arrive();
    for (int s = 0; s < a.steps; ++s) {
        const int cur = s & 1;
        const T* U = sm + (2 * cur) * PL;
        const T* V = U + PL;
        T* Un = sm + (2 * (cur ^ 1)) * PL;
        T* Vn = Un + PL;
        if (trace && s % trace_every == 0) {
            T* dst = trace + (size_t)(2 * (s / trace_every)) * NN + r0 * N;
            for (int i = tid; i < rp * N; i += nthr) {
                dst[i] = U[N + i];
                dst[NN + i] = V[N + i];
            }
        }
        if (ilo <= ihi) {
            for (int c = threadIdx.x; c < N; c += BX) {
                const int cl_ = (c + N - 1) & (N - 1), cr = (c + 1) & (N - 1);
                T uU = U[(ilo - 1) * N + c], vU = V[(ilo - 1) * N + c];
                T uC = U[ilo * N + c], vC = V[ilo * N + c];
                for (int r = ilo; r <= ihi; ++r) {
                    const int o = r * N;
                    const T uD = U[o + N + c], vD = V[o + N + c];
                    gs_update(k, uU, uC, uD, U[o + cl_], U[o + cr], vU, vC, vD, V[o + cl_], V[o + cr], &Un[o + c],
                              &Vn[o + c]);
                    uU = uC; uC = uD;
                    vU = vC; vC = vD;
                }
            }
        }
        cluster_wait();
        {
            const T* Uu = cl.map_shared_rank(U, up);
            const T* Vu = cl.map_shared_rank(V, up);
            const T* Ud = cl.map_shared_rank(U, down);
            const T* Vd = cl.map_shared_rank(V, down);
            for (int i = tid; i < 2 * N; i += nthr) {
                const int e = i / N, c = i & (N - 1);
                const int r = e == 0 ? 1 : rp;
                if (e == 1 && rp == 1) continue;
                const int cl_ = (c + N - 1) & (N - 1), cr = (c + 1) & (N - 1);
                const int o = r * N;
                const T uU = r == 1 ? Uu[rp * N + c] : U[o - N + c];
                const T vU = r == 1 ? Vu[rp * N + c] : V[o - N + c];
                const T uD = r == rp ? Ud[N + c] : U[o + N + c];
                const T vD = r == rp ? Vd[N + c] : V[o + N + c];
                gs_update(k, uU, U[o + c], uD, U[o + cl_], U[o + cr], vU, V[o + c], vD, V[o + cl_], V[o + cr],
                          &Un[o + c], &Vn[o + c]);
            }
        }
        __syncthreads();
        cluster_arrive();
    }
    cluster_wait();
    const int fin = a.steps & 1;
    for (int i = tid; i < rp * N; i += nthr) {
        uo[r0 * N + i] = sm[(2 * fin) * PL + N + i];
        vo[r0 * N + i] = sm[(2 * fin + 1) * PL + N + i];
    }
}

// Adjoint update of one cell (the transpose of gs_update): (aX, bX) the adjoint
// after the step around the cell, (uX, vX) the step's input state.  Adds the cell's
// contributions to the parameter gradients, before the dt factor and signs, to t:
//   t0 += a (1 - u), t1 += b v, t2 += a lap u, t3 += b lap v,
//   t4 += a (uR - uL) + b (vR - vL), t5 += a (uD - uU) + b (vD - vU)
// so that dL/dF = dt (t0 - t1), dL/dk = -dt t1, dL/dDu = dt t2, dL/dDv = dt t3,
// dL/dvx = -dt t4 / 2, dL/dvy = -dt t5 / 2.
template <typename T>
__device__ __forceinline__ void gs_adj_update(const GSCoef<T>& k, T aU, T aC, T aD, T aL, T aR, T bU, T bC, T bD,
                                              T bL, T bR, T uU, T uC, T uD, T uL, T uR, T vU, T vC, T vD, T vL,
                                              T vR, T* an, T* bn, T t[6]) {
    const T lap_a = fma(T(-4), aC, (aL + aR) + (aU + aD));
    const T lap_b = fma(T(-4), bC, (bL + bR) + (bU + bD));
    const T ba = bC - aC;
    T x = fma(k.du, lap_a, -k.dtF * aC);
    T y = fma(k.dv, lap_b, -k.dtFk * bC);
    if (k.drift) {
        x = fma(k.hx, aR - aL, fma(k.hy, aD - aU, x));
        y = fma(k.hx, bR - bL, fma(k.hy, bD - bU, y));
    }
    x = fma(k.dt * (vC * vC), ba, x);
    y = fma((k.dt + k.dt) * (uC * vC), ba, y);
    *an = aC + x;
    *bn = bC + y;
    const T lu = fma(T(-4), uC, (uL + uR) + (uU + uD));
    const T lv = fma(T(-4), vC, (vL + vR) + (vU + vD));
    t[0] = fma(aC, T(1) - uC, t[0]);
    t[1] = fma(bC, vC, t[1]);
    t[2] = fma(aC, lu, t[2]);
    t[3] = fma(bC, lv, t[3]);
    t[4] = fma(aC, uR - uL, fma(bC, vR - vL, t[4]));
    t[5] = fma(aC, uD - uU, fma(bC, vD - vU, t[5]));
}

__device__ __forceinline__ void grad_finish(const double g[6], double dt, double out[6]) {
    out[0] = dt * (g[0] - g[1]);
    out[1] = -dt * g[1];
    out[2] = dt * g[2];
    out[3] = dt * g[3];
    out[4] = -0.5 * dt * g[4];
    out[5] = -0.5 * dt * g[5];
}

// block-reduce the six per-thread gradient sums and add them to grad[0..5]
__device__ __forceinline__ void grad_reduce(const double g[6], double dt, double* grad, double (*red)[32], int tid,
                                            int nthr) {
    double o[6];
    grad_finish(g, dt, o);
#pragma unroll
    for (int q = 0; q < 6; ++q) {
        double v = o[q];
        for (int s = 16; s > 0; s >>= 1) v += __shfl_xor_sync(0xffffffffu, v, s);
        if ((tid & 31) == 0) red[q][tid >> 5] = v;
    }
    __syncthreads();
    if (tid < 6) {
        double v = 0;
        for (int w = 0; w < nthr / 32; ++w) v += red[tid][w];
        atomicAdd(&grad[tid], v);
    }
}

template <typename T, int N>
__global__ void __launch_bounds__(512, 1) k_gs_adjoint_cw(GSArgs<T> a, const T* __restrict__ states, int len,
                                                         const T* __restrict__ lu_in, const T* __restrict__ lv_in,
                                                         T* __restrict__ lu_out, T* __restrict__ lv_out,
                                                         double* __restrict__ grad, int* __restrict__ err) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* sm = reinterpret_cast<T*>(smem_raw);
    __shared__ double red[6][32];
    cg::cluster_group cl = cg::this_cluster();
    const int rp = N / (int)cl.num_blocks();
    const int r0 = (int)cl.block_rank() * rp;
    constexpr int NN = N * N;
    const int BX = blockDim.x, BY = blockDim.y;
    const int tid = threadIdx.y * BX + threadIdx.x;
    const int nthr = BX * BY;
    const int rpt = rp / BY;
    const int rb = 1 + threadIdx.y * rpt;
    const int ilo = rb < 2 ? 2 : rb;
    const int ihi = rb + rpt - 1 > rp - 1 ? rp - 1 : rb + rpt - 1;
    const unsigned rank = cl.block_rank(), nb = cl.num_blocks();
    const unsigned up = (rank + nb - 1) % nb, down = (rank + 1) % nb;
    const GSCoef<T> k(a);
    (void)err;
    const int PL = (rp + 2) * N;
    for (int i = tid; i < rp * N; i += nthr) {
        sm[N + i] = lu_in[r0 * N + i];
        sm[PL + N + i] = lv_in[r0 * N + i];
    }
    double g[6] = {0, 0, 0, 0, 0, 0};
    __syncthreads();
    cluster_arrive();
    for (int j = len - 1, s = 0; j >= 0; --j, ++s) {
        const int cur = s & 1;
        const T* A = sm + (2 * cur) * PL;
        const T* B = A + PL;
        T* An = sm + (2 * (cur ^ 1)) * PL;
        T* Bn = An + PL;
        const T* Us = states + (size_t)(2 * j) * NN;
        const T* Vs = Us + NN;
        T t[6] = {T(0), T(0), T(0), T(0), T(0), T(0)};
        if (ilo <= ihi) {
            for (int c = threadIdx.x; c < N; c += BX) {
                const int cl_ = (c + N - 1) & (N - 1), cr = (c + 1) & (N - 1);
                const int g0 = r0 + ilo - 1;
                T uU = Us[(g0 - 1) * N + c], vU = Vs[(g0 - 1) * N + c];
                T uC = Us[g0 * N + c], vC = Vs[g0 * N + c];
                T aU = A[(ilo - 1) * N + c], bU = B[(ilo - 1) * N + c];
                T aC = A[ilo * N + c], bC = B[ilo * N + c];
                for (int r = ilo; r <= ihi; ++r) {
                    const int o = r * N, go = (r0 + r - 1) * N;
                    const T uD = Us[go + N + c], vD = Vs[go + N + c];
                    const T aD = A[o + N + c], bD = B[o + N + c];
                    gs_adj_update(k, aU, aC, aD, A[o + cl_], A[o + cr], bU, bC, bD, B[o + cl_], B[o + cr], uU, uC, uD,
                                  Us[go + cl_], Us[go + cr], vU, vC, vD, Vs[go + cl_], Vs[go + cr], &An[o + c],
                                  &Bn[o + c], t);
                    uU = uC; uC = uD; vU = vC; vC = vD;
                    aU = aC; aC = aD; bU = bC; bC = bD;
                }
            }
        }
        cluster_wait();
        {
            const T* Au = cl.map_shared_rank(A, up);
            const T* Bu = cl.map_shared_rank(B, up);
            const T* Ad = cl.map_shared_rank(A, down);
            const T* Bd = cl.map_shared_rank(B, down);
            for (int i = tid; i < 2 * N; i += nthr) {
                const int e = i / N, c = i & (N - 1);
                const int r = e == 0 ? 1 : rp;
                if (e == 1 && rp == 1) continue;
                const int cl_ = (c + N - 1) & (N - 1), cr = (c + 1) & (N - 1);
                const int o = r * N;
                const int gr = r0 + r - 1;
                const int gu = (gr + N - 1) & (N - 1), gd = (gr + 1) & (N - 1);
                const int go = gr * N;
                const T aU = r == 1 ? Au[rp * N + c] : A[o - N + c];
                const T bU = r == 1 ? Bu[rp * N + c] : B[o - N + c];
                const T aD = r == rp ? Ad[N + c] : A[o + N + c];
                const T bD = r == rp ? Bd[N + c] : B[o + N + c];
                gs_adj_update(k, aU, A[o + c], aD, A[o + cl_], A[o + cr], bU, B[o + c], bD, B[o + cl_], B[o + cr],
                              Us[gu * N + c], Us[go + c], Us[gd * N + c], Us[go + cl_], Us[go + cr],
                              Vs[gu * N + c], Vs[go + c], Vs[gd * N + c], Vs[go + cl_], Vs[go + cr],
                              &An[o + c], &Bn[o + c], t);
            }
        }
#pragma unroll
        for (int q = 0; q < 6; ++q) g[q] += (double)t[q];
        __syncthreads();
        cluster_arrive();
    }
    cluster_wait();
    const int fin = len & 1;
    for (int i = tid; i < rp * N; i += nthr) {
        lu_out[r0 * N + i] = sm[(2 * fin) * PL + N + i];
        lv_out[r0 * N + i] = sm[(2 * fin + 1) * PL + N + i];
    }
    grad_reduce(g, (double)a.dt, grad, red, tid, nthr);
}

#include "gs_f32x2.cuh"
#include "gs_rr.cuh"
#include "gs_mc.cuh"

// register-resident forward kernel for an n x n float32 lattice with *wpc warps per
// CTA (*wpc = 0: the default split, written back), or NULL where the lattice does
// not fit it
const void* rr_kernel(int n, int* wpc, bool drift, size_t* smem) {
#define GS_RR_CASE(N_, W_)                                                                        \
    if (n == N_ && *wpc == W_) {                                                                  \
        *smem = RRShape<N_, W_>::kSmem;                                                           \
        return drift ? (const void*)k_gs_forward_rr<N_, W_, 1> : (const void*)k_gs_forward_rr<N_, W_, 0>; \
    }
    if (*wpc == 0) *wpc = n == 256 ? 8 : n == 128 ? 4 : 2;
    GS_RR_CASE(64, 1) GS_RR_CASE(64, 2) GS_RR_CASE(64, 4)
    GS_RR_CASE(128, 2) GS_RR_CASE(128, 4) GS_RR_CASE(128, 8)
    GS_RR_CASE(256, 4) GS_RR_CASE(256, 8) GS_RR_CASE(256, 16)
#undef GS_RR_CASE
    return nullptr;
}

// Multi-cluster forward kernels (gs_mc.cuh): variant 40 + index.  Each spreads one
// lattice over `clusters` 16-CTA clusters with `ghost` ghost rows per band side.
struct MCConfig {
    int n, clusters, ghost, wpc;
    const void* k[2][2];   // [forward / adjoint][without / with drift]
    uint32_t smem;
    size_t xwords;   // exchange buffer, 64-bit words
};
template <int N, int C, int G, int W>
MCConfig mc_config() {
    using S = MCShape<N, C, G, W>;
    return {N, C, G, W,
            {{(const void*)k_gs_forward_mc<N, C, G, W, 0>, (const void*)k_gs_forward_mc<N, C, G, W, 1>},
             {(const void*)k_gs_adjoint_mc<N, C, G, W, 0>, (const void*)k_gs_adjoint_mc<N, C, G, W, 1>}},
            S::kSmem, S::kXWords};
}
constexpr int kMCVariant = 40;
constexpr int kMCConfigs = 7;
// the automatic choice for n = 256: 4 clusters, 8 ghost rows (0.587 us per step;
// (4, 16) 0.594, (4, 32) 0.611, the single-cluster kernel 0.74)
constexpr int kMCDefault = 1;
const MCConfig& mc_table(int i) {
    static const MCConfig t[kMCConfigs] = {mc_config<256, 2, 8, 9>(),   mc_config<256, 4, 8, 5>(),
                                           mc_config<256, 4, 16, 6>(),  mc_config<256, 8, 8, 3>(),
                                           mc_config<256, 8, 16, 4>(),  mc_config<256, 4, 32, 8>(),
                                           mc_config<256, 2, 32, 12>()};
    return t[i];
}

// launch configuration of a multi-cluster kernel.  The clusters wait on one another's
// rows, so all of them must be resident at once: mc_fits checks that the device holds
// them (the launch itself is not cooperative, which the profiler refuses for cluster
// launches), and every wait is bounded, so a cluster that is not running yet costs a
// NaN result and an error status, never a hang
void mc_launch_config(const MCConfig& m, cudaLaunchConfig_t* cfg, cudaLaunchAttribute* attr, cudaStream_t st) {
    *cfg = {};
    cfg->gridDim = dim3(kRRCluster * m.clusters, 1, 1);
    cfg->blockDim = dim3(32 * m.wpc, 1, 1);
    cfg->dynamicSmemBytes = m.smem;
    cfg->stream = st;
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = kRRCluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg->attrs = attr;
    cfg->numAttrs = 1;
}

// whether every cluster of configuration i can be resident at once on the current
// device (the kernel spins on the other clusters' flags), cached per device
cudaError_t mc_fits(int i, bool drift, bool* fits, int kind = 0) {
    static int cache[64][kMCConfigs][2][2];   // [dev][config][forward / adjoint][drift]: 0 unknown, 1 fits, 2 not
    static std::mutex mu;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) {
        *fits = false;
        return cudaSuccess;
    }
    std::lock_guard<std::mutex> lock(mu);
    int& c = cache[dev][i][kind][drift ? 1 : 0];
    if (c == 0) {
        const MCConfig& m = mc_table(i);
        const void* fn = m.k[kind][drift ? 1 : 0];
        e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)m.smem);
        if (e == cudaSuccess) e = cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        if (e != cudaSuccess) return e;
        cudaLaunchConfig_t cfg;
        cudaLaunchAttribute attr[1];
        mc_launch_config(m, &cfg, attr, nullptr);
        int active = 0;
        e = cudaOccupancyMaxActiveClusters(&active, fn, &cfg);
        if (e != cudaSuccess) return e;
        c = active >= m.clusters ? 1 : 2;
    }
    *fits = c == 1;
    return cudaSuccess;
}

// one multi-cluster launch (kind 0 forward, 1 adjoint segment): exchange buffer from
// the stream-ordered pool (private to this launch), cleared on the stream, then the
// kernel with `args` followed by the buffer pointer
cudaError_t mc_run(int i, int kind, bool drift, void** args, int nargs, cudaStream_t st) {
    const MCConfig& m = mc_table(i);
    const void* fn = m.k[kind][drift ? 1 : 0];
    const size_t xbytes = m.xwords * sizeof(uint64_t);
    uint64_t* xb = nullptr;
    cudaError_t e = pool_alloc((void**)&xb, xbytes, st);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(xb, 0, xbytes, st);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)m.smem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    if (e == cudaSuccess) {
        void* all[16];
        for (int q = 0; q < nargs; ++q) all[q] = args[q];
        all[nargs] = &xb;
        cudaLaunchConfig_t cfg;
        cudaLaunchAttribute attr[1];
        mc_launch_config(m, &cfg, attr, st);
        e = cudaLaunchKernelExC(&cfg, fn, all);
    }
    cudaError_t e2 = pool_free(xb, st);
    return e != cudaSuccess ? e : e2;
}

cudaError_t mc_forward(int i, const GSArgs<float>& a0, bool drift, const float* u0, const float* v0, float* u,
                       float* v, float* trace, int every, cudaStream_t st) {
    GSArgs<float> a = a0;
    void* args[] = {&a, (void*)&u0, (void*)&v0, &u, &v, &trace, &every};
    return mc_run(i, 0, drift, args, 7, st);
}

// register-resident adjoint kernel with wpc warps per CTA
const void* rr_adj_kernel(int n, int* wpc, bool drift, size_t* smem) {
#define GS_RRA_CASE(N_, W_)                                                                        \
    if (n == N_ && *wpc == W_) {                                                                   \
        *smem = RRAdjShape<N_, W_>::kSmem;                                                         \
        return drift ? (const void*)k_gs_adjoint_rr<N_, W_, 1> : (const void*)k_gs_adjoint_rr<N_, W_, 0>; \
    }
    if (*wpc == 0) *wpc = n == 256 ? 8 : n == 128 ? 4 : 2;
    GS_RRA_CASE(64, 1) GS_RRA_CASE(64, 2) GS_RRA_CASE(64, 4)
    GS_RRA_CASE(128, 2) GS_RRA_CASE(128, 4) GS_RRA_CASE(128, 8)
    GS_RRA_CASE(256, 4) GS_RRA_CASE(256, 8)
#undef GS_RRA_CASE
    return nullptr;
}

template <typename T>
const void* fwd_kernel(int n) {
    if (sizeof(T) == 4) {
        switch (n) {
            case 64: return (const void*)k_gs_forward_x2<64>;
            case 128: return (const void*)k_gs_forward_x2<128>;
            case 256: return (const void*)k_gs_forward_x2<256>;
            case 512: return (const void*)k_gs_forward_x2<512>;
            default: return nullptr;
        }
    }
    switch (n) {
        case 64: return (const void*)k_gs_forward_cw<T, 64>;
        case 128: return (const void*)k_gs_forward_cw<T, 128>;
        case 256: return (const void*)k_gs_forward_cw<T, 256>;
        case 512: return (const void*)k_gs_forward_cw<T, 512>;
        default: return nullptr;
    }
}
template <typename T>
const void* adj_kernel(int n) {
    if (sizeof(T) == 4) {
        switch (n) {
            case 64: return (const void*)k_gs_adjoint_x2<64>;
            case 128: return (const void*)k_gs_adjoint_x2<128>;
            case 256: return (const void*)k_gs_adjoint_x2<256>;
            case 512: return (const void*)k_gs_adjoint_x2<512>;
            default: return nullptr;
        }
    }
    switch (n) {
        case 64: return (const void*)k_gs_adjoint_cw<T, 64>;
        case 128: return (const void*)k_gs_adjoint_cw<T, 128>;
        case 256: return (const void*)k_gs_adjoint_cw<T, 256>;
        case 512: return (const void*)k_gs_adjoint_cw<T, 512>;
        default: return nullptr;
    }
}

// Block shape of the packed float32 kernels: BX column pairs, rows split evenly.
dim3 x2_block(int n, int cluster, int max_threads) {
    const int bx = n / 2 < 256 ? n / 2 : 256;
    if (bx < 32 || (n / 2) % bx) return dim3(0, 0, 1);
    const int rp = n / cluster;
    int by = max_threads / bx;
    while (by > 1 && rp % by) by >>= 1;
    if (rp % by) return dim3(0, 0, 1);
    return dim3(bx, by, 1);
}

template <typename T>
cudaError_t launch_cluster(const void* fn, int n, int cluster, size_t smem, cudaStream_t st, void** args,
                           dim3 block = dim3(kThreads, 1, 1)) {
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    if (cluster > 8) {
        e = cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        if (e != cudaSuccess) return e;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(cluster, 1, 1);
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    (void)n;
    return cudaLaunchKernelExC(&cfg, fn, args);
}

template <typename T>
size_t smem_bytes(int n, int cluster) {
    return sizeof(T) * 2 * 2 * (size_t)(n / cluster + 2) * n;
}

// Block shape of the column-walk kernels, or bx = 0 when the lattice does not fit
// their layout (n a multiple of 32, the CTA's rows split evenly across block rows).
dim3 cw_block(int n, int cluster, int max_threads = 1024) {
    if (n % 32 != 0) return dim3(0, 0, 1);
    const int bx = n < 256 ? n : 256;
    if (n % bx) return dim3(0, 0, 1);
    const int rp = n / cluster;
    int by = max_threads / bx;
    while (by > 1 && rp % by) by >>= 1;
    if (rp % by) return dim3(0, 0, 1);
    return dim3(bx, by, 1);
}

}  // namespace

int gs_cluster_size(int n, int elem_bytes) {
    // 16 CTAs (16 SMs) when the lattice splits into 16 slabs that fit, else the
    // smallest cluster that holds the lattice in shared memory
    if (n % 16 == 0 && (size_t)elem_bytes * 4 * (size_t)(n / 16 + 2) * n <= 200 * 1024 && cw_block(n, 16).x != 0)
        return 16;
    for (int c : {1, 2, 4, 8, 16}) {
        if (n % c) continue;
        if ((size_t)elem_bytes * 4 * (size_t)(n / c + 2) * n <= 200 * 1024) return c;
    }
    return 0;
}

template <typename T>
cudaError_t gs_forward(const GSParams& p, const T* u0, const T* v0, T* u, T* v, T* trace, int trace_every,
                       cudaStream_t st) {
    const int cl = p.cluster > 0 ? p.cluster : gs_cluster_size(p.n, (int)sizeof(T));
    if (cl <= 0) return cudaErrorInvalidValue;
    GSArgs<T> a{p.n, p.steps, (T)p.F, (T)p.k, (T)p.Du, (T)p.Dv, (T)p.vx, (T)p.vy, (T)p.dt};
    int every = trace_every > 0 ? trace_every : 1;
    void* args[] = {&a, (void*)&u0, (void*)&v0, &u, &v, &trace, &every};
    if constexpr (std::is_same<T, float>::value) {
        const bool drift = p.vx != 0.0 || p.vy != 0.0;
        if (p.variant >= kMCVariant && p.variant < kMCVariant + kMCConfigs) {
            const int i = p.variant - kMCVariant;
            bool fits = false;
            if (cl != kRRCluster || mc_table(i).n != p.n) return cudaErrorInvalidValue;
            cudaError_t e = mc_fits(i, drift, &fits);
            if (e != cudaSuccess) return e;
            if (!fits) return cudaErrorInvalidConfiguration;
            return mc_forward(i, a, drift, u0, v0, u, v, trace, every, st);
        }
        if (p.variant == 0 && cl == kRRCluster && p.n == mc_table(kMCDefault).n) {
            bool fits = false;
            cudaError_t e = mc_fits(kMCDefault, drift, &fits);
            if (e != cudaSuccess) return e;
            if (fits) return mc_forward(kMCDefault, a, drift, u0, v0, u, v, trace, every, st);
        }
    }
    if (sizeof(T) == 4 && cl == kRRCluster && (p.variant == 0 || p.variant == 3 || (p.variant > 10 && p.variant < kMCVariant))) {
        size_t smem = 0;
        int wpc = p.variant > 10 ? p.variant - 10 : 0;
        const void* rk = rr_kernel(p.n, &wpc, p.vx != 0.0 || p.vy != 0.0, &smem);
        const GSArgs<float>* no_batch = nullptr;
        void* rargs[] = {&a, (void*)&u0, (void*)&v0, &u, &v, &trace, &every, &no_batch};
        if (rk) return launch_cluster<T>(rk, p.n, cl, smem, st, rargs, dim3(32 * wpc, 1, 1));
        if (p.variant != 0) return cudaErrorInvalidValue;
    }
    const dim3 blk = sizeof(T) == 4 ? x2_block(p.n, cl, 512) : cw_block(p.n, cl);
    const void* fk = fwd_kernel<T>(p.n);
    if (blk.x != 0 && fk && p.variant != 1) return launch_cluster<T>(fk, p.n, cl, smem_bytes<T>(p.n, cl), st, args, blk);
    return launch_cluster<T>((const void*)k_gs_forward<T>, p.n, cl, smem_bytes<T>(p.n, cl), st, args);
}

template <typename T>
cudaError_t gs_adjoint_segment(const GSParams& p, const T* states, int len, const T* lu_in, const T* lv_in, T* lu_out,
                               T* lv_out, double* grad, int* err, cudaStream_t st) {
    const int cl = p.cluster > 0 ? p.cluster : gs_cluster_size(p.n, (int)sizeof(T));
    if (cl <= 0) return cudaErrorInvalidValue;
    GSArgs<T> a{p.n, p.steps, (T)p.F, (T)p.k, (T)p.Du, (T)p.Dv, (T)p.vx, (T)p.vy, (T)p.dt};
    void* args[] = {&a, (void*)&states, &len, (void*)&lu_in, (void*)&lv_in, &lu_out, &lv_out, &grad, &err};
    if constexpr (std::is_same<T, float>::value) {
        // the multi-cluster adjoint, with a multi-cluster variant only (the gradient
        // pipeline names it under the automatic choice, with the single-cluster forward
        // recomputing the segments beside it: two 64-SM kernels at once made the
        // backward slower, 18.1 ms against 15.4 ms)
        const bool drift = p.vx != 0.0 || p.vy != 0.0;
        int i = -1;
        if (p.variant >= kMCVariant && p.variant < kMCVariant + kMCConfigs) i = p.variant - kMCVariant;
        if (i >= 0 && cl == kRRCluster && mc_table(i).n == p.n) {
            bool fits = false;
            cudaError_t e = mc_fits(i, drift, &fits, 1);
            if (e != cudaSuccess) return e;
            if (fits) return mc_run(i, 1, drift, args, 9, st);
            if (p.variant != 0) return cudaErrorInvalidConfiguration;
        }
    }
    const int variant = p.variant >= kMCVariant ? 0 : p.variant;
    if (sizeof(T) == 4 && cl == kRRCluster && (variant == 0 || variant == 3 || variant > 10)) {
        size_t smem = 0;
        int wpc = variant > 10 ? variant - 10 : 0;
        const void* rk = rr_adj_kernel(p.n, &wpc, p.vx != 0.0 || p.vy != 0.0, &smem);
        if (rk) return launch_cluster<T>(rk, p.n, cl, smem, st, args, dim3(32 * wpc, 1, 1));
        if (variant != 0) return cudaErrorInvalidValue;
    }
    const dim3 blk = sizeof(T) == 4 ? x2_block(p.n, cl, 512) : cw_block(p.n, cl, 512);
    const void* ak = adj_kernel<T>(p.n);
    // the packed float32 adjoint also holds two state buffers in shared memory
    const size_t smem = smem_bytes<T>(p.n, cl) * (sizeof(T) == 4 ? 2 : 1);
    if (blk.x != 0 && ak && p.variant != 1) return launch_cluster<T>(ak, p.n, cl, smem, st, args, blk);
    return launch_cluster<T>((const void*)k_gs_adjoint<T>, p.n, cl, smem_bytes<T>(p.n, cl), st, args);
}

cudaError_t gs_forward_batch_f32(const GSParams& p, int batch, const GSBatchMember* members, const float* u0,
                                 const float* v0, float* u, float* v, cudaStream_t st) {
    if (batch <= 0 || !members) return cudaErrorInvalidValue;
    bool drift = false;
    std::vector<GSArgs<float>> h(batch);
    for (int b = 0; b < batch; ++b) {
        const GSBatchMember& m = members[b];
        h[b] = GSArgs<float>{p.n, p.steps, (float)m.F, (float)m.k, (float)m.Du, (float)m.Dv, (float)m.vx, (float)m.vy,
                             (float)p.dt};
        drift = drift || m.vx != 0.0 || m.vy != 0.0;
    }
    size_t smem = 0;
    int wpc = p.variant > 10 && p.variant < kMCVariant ? p.variant - 10 : 0;   // one lattice per cluster
    const void* rk = rr_kernel(p.n, &wpc, drift, &smem);
    if (!rk) return cudaErrorInvalidValue;
    GSArgs<float>* d = nullptr;
    cudaError_t e = pool_alloc((void**)&d, sizeof(GSArgs<float>) * batch, st);
    if (e != cudaSuccess) return e;
    e = cudaMemcpyAsync(d, h.data(), sizeof(GSArgs<float>) * batch, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        GSArgs<float> a = h[0];
        float* no_trace = nullptr;
        int every = 1;
        void* args[] = {&a, (void*)&u0, (void*)&v0, &u, &v, &no_trace, &every, &d};
        e = cudaFuncSetAttribute(rk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e == cudaSuccess) e = cudaFuncSetAttribute(rk, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        if (e == cudaSuccess) {
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3(kRRCluster * batch, 1, 1);
            cfg.blockDim = dim3(32 * wpc, 1, 1);
            cfg.dynamicSmemBytes = smem;
            cfg.stream = st;
            cudaLaunchAttribute attr[1];
            attr[0].id = cudaLaunchAttributeClusterDimension;
            attr[0].val.clusterDim.x = kRRCluster;
            attr[0].val.clusterDim.y = 1;
            attr[0].val.clusterDim.z = 1;
            cfg.attrs = attr;
            cfg.numAttrs = 1;
            e = cudaLaunchKernelExC(&cfg, rk, args);
        }
    }
    cudaError_t e2 = pool_free(d, st);
    return e != cudaSuccess ? e : e2;
}

cudaError_t gs_auto_variant(int n, bool drift, int* variant) {
    const int cl = gs_cluster_size(n, 4);
    if (cl == kRRCluster && n == mc_table(kMCDefault).n) {
        bool fits = false;
        cudaError_t e = mc_fits(kMCDefault, drift, &fits);
        if (e != cudaSuccess) return e;
        if (fits) {
            *variant = kMCVariant + kMCDefault;
            return cudaSuccess;
        }
    }
    size_t smem = 0;
    int wpc = 0;
    if (cl == kRRCluster && rr_kernel(n, &wpc, drift, &smem)) {
        *variant = 10 + wpc;
        return cudaSuccess;
    }
    *variant = cl > 0 && x2_block(n, cl, 512).x != 0 && fwd_kernel<float>(n) ? 2 : 1;
    return cudaSuccess;
}

cudaError_t gs_batch_capacity(int n, int* clusters) {
    size_t smem = 0;
    int wpc = 0;
    const void* rk = rr_kernel(n, &wpc, false, &smem);
    if (!rk) return cudaErrorInvalidValue;
    cudaError_t e = cudaFuncSetAttribute(rk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(rk, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(kRRCluster, 1, 1);
    cfg.blockDim = dim3(32 * wpc, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = kRRCluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaOccupancyMaxActiveClusters(clusters, rk, &cfg);
}

cudaError_t gs_forward_status(int* out, bool clear) {
    int v = 0;
    cudaError_t e = cudaMemcpyFromSymbol(&v, g_gs_fwd_err, sizeof(int));
    if (e != cudaSuccess) return e;
    if (clear && v) {
        const int zero = 0;
        e = cudaMemcpyToSymbol(g_gs_fwd_err, &zero, sizeof(int));
        if (e != cudaSuccess) return e;
    }
    *out = v;
    return cudaSuccess;
}

template cudaError_t gs_forward<float>(const GSParams&, const float*, const float*, float*, float*, float*, int,
                                       cudaStream_t);
template cudaError_t gs_forward<double>(const GSParams&, const double*, const double*, double*, double*, double*, int,
                                        cudaStream_t);
template cudaError_t gs_adjoint_segment<float>(const GSParams&, const float*, int, const float*, const float*, float*,
                                               float*, double*, int*, cudaStream_t);
template cudaError_t gs_adjoint_segment<double>(const GSParams&, const double*, int, const double*, const double*,
                                                double*, double*, double*, int*, cudaStream_t);

}  // namespace gpgmp
