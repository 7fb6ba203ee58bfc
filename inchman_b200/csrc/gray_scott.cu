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
#include <cuda_runtime.h>
#include "gs_kernels.h"

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
                                                           double* __restrict__ grad) {
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

template <typename T>
cudaError_t launch_cluster(const void* fn, int n, int cluster, size_t smem, cudaStream_t st, void** args) {
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    if (cluster > 8) {
        e = cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        if (e != cudaSuccess) return e;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(cluster, 1, 1);
    cfg.blockDim = dim3(kThreads, 1, 1);
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

}  // namespace

int gs_cluster_size(int n, int elem_bytes) {
    // the smallest cluster (<= 16) that fits the lattice in shared memory
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
    return launch_cluster<T>((const void*)k_gs_forward<T>, p.n, cl, smem_bytes<T>(p.n, cl), st, args);
}

template <typename T>
cudaError_t gs_adjoint_segment(const GSParams& p, const T* states, int len, const T* lu_in, const T* lv_in, T* lu_out,
                               T* lv_out, double* grad, cudaStream_t st) {
    const int cl = p.cluster > 0 ? p.cluster : gs_cluster_size(p.n, (int)sizeof(T));
    if (cl <= 0) return cudaErrorInvalidValue;
    GSArgs<T> a{p.n, p.steps, (T)p.F, (T)p.k, (T)p.Du, (T)p.Dv, (T)p.vx, (T)p.vy, (T)p.dt};
    void* args[] = {&a, (void*)&states, &len, (void*)&lu_in, (void*)&lv_in, &lu_out, &lv_out, &grad};
    return launch_cluster<T>((const void*)k_gs_adjoint<T>, p.n, cl, smem_bytes<T>(p.n, cl), st, args);
}

template cudaError_t gs_forward<float>(const GSParams&, const float*, const float*, float*, float*, float*, int,
                                       cudaStream_t);
template cudaError_t gs_forward<double>(const GSParams&, const double*, const double*, double*, double*, double*, int,
                                        cudaStream_t);
template cudaError_t gs_adjoint_segment<float>(const GSParams&, const float*, int, const float*, const float*, float*,
                                               float*, double*, cudaStream_t);
template cudaError_t gs_adjoint_segment<double>(const GSParams&, const double*, int, const double*, const double*,
                                                double*, double*, double*, cudaStream_t);

}  // namespace gpgmp
