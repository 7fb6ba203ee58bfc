// Float32 Gray-Scott kernels built on Blackwell's packed FP32x2 instructions
// (__ffma2_rn / __fadd2_rn / __fmul2_rn): a thread owns a pair of adjacent
// columns and updates both cells with one packed instruction per operation, which
// halves the issue slots of the arithmetic.  Same cluster structure as the scalar
// kernels (slabs in shared memory, split-phase cluster barrier, DSMEM edge rows).
// The adjoint additionally prefetches the next step's stored state rows into shared
// memory with TMA bulk copies (cp.async.bulk, completion on an mbarrier) while the
// current step is computed.
//
// Included from gray_scott.cu (uses GSArgs, cluster_arrive / cluster_wait,
// grad_reduce).

__device__ __forceinline__ float2 f2(float x) { return make_float2(x, x); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(make_float2(-1.f, -1.f), b, a); }
__device__ __forceinline__ float2 ld2(const float* p) { return *reinterpret_cast<const float2*>(p); }
__device__ __forceinline__ void st2(float* p, float2 v) { *reinterpret_cast<float2*>(p) = v; }

struct GSCoef2 {
    float2 du, dv, hx, hy, dt, mdt, dtF, mdtF, mdtFk, m4, one, two_dt;
    bool drift;
    __device__ __forceinline__ explicit GSCoef2(const GSArgs<float>& a) {
        du = f2(a.dt * a.Du);
        dv = f2(a.dt * a.Dv);
        hx = f2(a.dt * a.vx * 0.5f);
        hy = f2(a.dt * a.vy * 0.5f);
        dt = f2(a.dt);
        mdt = f2(-a.dt);
        dtF = f2(a.dt * a.F);
        mdtF = f2(-(a.dt * a.F));
        mdtFk = f2(-(a.dt * (a.F + a.k)));
        m4 = f2(-4.f);
        one = f2(1.f);
        two_dt = f2(a.dt + a.dt);
        drift = a.vx != 0.f || a.vy != 0.f;
    }
};

// forward update of two cells at once: C the cells, L / R / U / D their left,
// right, upper and lower neighbours (any pairing of cells; the arithmetic per cell
// is the same as in the scalar kernels' gs_update).  DRIFT: 1 with the drift
// terms, 0 without, -1 decided by k.drift at run time.
template <int DRIFT = -1>
__device__ __forceinline__ void gs_update2f(const GSCoef2& k, float2 uL, float2 uR, float2 uU, float2 uC, float2 uD,
                                            float2 vL, float2 vR, float2 vU, float2 vC, float2 vD, float2* un,
                                            float2* vn) {
    const float2 uvv = mul2(uC, mul2(vC, vC));
    const float2 lu = fma2(k.m4, uC, add2(add2(uL, uR), add2(uU, uD)));
    const float2 lv = fma2(k.m4, vC, add2(add2(vL, vR), add2(vU, vD)));
    float2 a = fma2(k.du, lu, fma2(k.mdtF, uC, k.dtF));
    float2 b = fma2(k.mdtFk, vC, mul2(k.dv, lv));
    if (DRIFT == 1 || (DRIFT < 0 && k.drift)) {
        a = fma2(k.hx, sub2(uL, uR), fma2(k.hy, sub2(uU, uD), a));
        b = fma2(k.hx, sub2(vL, vR), fma2(k.hy, sub2(vU, vD), b));
    }
    *un = add2(uC, fma2(k.mdt, uvv, a));
    *vn = add2(vC, fma2(k.dt, uvv, b));
}

// forward update of the adjacent pair C = (x, x+1), L = (x-1, x), R = (x+1, x+2)
__device__ __forceinline__ void gs_update2(const GSCoef2& k, float2 uU, float2 uC, float2 uD, float uLs, float uRs,
                                           float2 vU, float2 vC, float2 vD, float vLs, float vRs, float2* un,
                                           float2* vn) {
    gs_update2f(k, make_float2(uLs, uC.x), make_float2(uC.y, uRs), uU, uC, uD, make_float2(vLs, vC.x),
                make_float2(vC.y, vRs), vU, vC, vD, un, vn);
}

template <int N>
__global__ void __launch_bounds__(512, 1) k_gs_forward_x2(GSArgs<float> a, const float* __restrict__ u0,
                                                         const float* __restrict__ v0, float* __restrict__ uo,
                                                         float* __restrict__ vo, float* __restrict__ trace,
                                                         int trace_every) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float* sm = reinterpret_cast<float*>(smem_raw);
    cg::cluster_group cl = cg::this_cluster();
    const int rp = N / (int)cl.num_blocks();
    const int r0 = (int)cl.block_rank() * rp;
    constexpr int NN = N * N;
    const int BX = blockDim.x, BY = blockDim.y;   // BX pairs of columns
    const int tid = threadIdx.y * BX + threadIdx.x;
    const int nthr = BX * BY;
    const int rpt = rp / BY;
    const int rb = 1 + threadIdx.y * rpt;
    const int ilo = rb < 2 ? 2 : rb;
    const int ihi = rb + rpt - 1 > rp - 1 ? rp - 1 : rb + rpt - 1;
    const unsigned rank = cl.block_rank(), nb = cl.num_blocks();
    const unsigned up = (rank + nb - 1) % nb, down = (rank + 1) % nb;
    const GSCoef2 k(a);
    const int PL = (rp + 2) * N;
    for (int i = tid; i < rp * N / 4; i += nthr) {
        reinterpret_cast<float4*>(sm + N)[i] = reinterpret_cast<const float4*>(u0 + r0 * N)[i];
        reinterpret_cast<float4*>(sm + PL + N)[i] = reinterpret_cast<const float4*>(v0 + r0 * N)[i];
    }
    __syncthreads();
    cluster_arrive();
    for (int s = 0; s < a.steps; ++s) {
        const int cur = s & 1;
        const float* U = sm + (2 * cur) * PL;
        const float* V = U + PL;
        float* Un = sm + (2 * (cur ^ 1)) * PL;
        float* Vn = Un + PL;
        if (trace && s % trace_every == 0) {
            float* dst = trace + (size_t)(2 * (s / trace_every)) * NN + r0 * N;
            for (int i = tid; i < rp * N / 4; i += nthr) {
                reinterpret_cast<float4*>(dst)[i] = reinterpret_cast<const float4*>(U + N)[i];
                reinterpret_cast<float4*>(dst + NN)[i] = reinterpret_cast<const float4*>(V + N)[i];
            }
        }
        if (ilo <= ihi) {
            for (int p = threadIdx.x; p < N / 2; p += BX) {
                const int c = 2 * p;
                const int cl_ = (c + N - 1) & (N - 1), cr = (c + 2) & (N - 1);
                float2 uU = ld2(U + (ilo - 1) * N + c), vU = ld2(V + (ilo - 1) * N + c);
                float2 uC = ld2(U + ilo * N + c), vC = ld2(V + ilo * N + c);
                for (int r = ilo; r <= ihi; ++r) {
                    const int o = r * N;
                    const float2 uD = ld2(U + o + N + c), vD = ld2(V + o + N + c);
                    float2 un, vn;
                    gs_update2(k, uU, uC, uD, U[o + cl_], U[o + cr], vU, vC, vD, V[o + cl_], V[o + cr], &un, &vn);
                    st2(Un + o + c, un);
                    st2(Vn + o + c, vn);
                    uU = uC; uC = uD;
                    vU = vC; vC = vD;
                }
            }
        }
        cluster_wait();
        {
            const float* Uu = cl.map_shared_rank(U, up);
            const float* Vu = cl.map_shared_rank(V, up);
            const float* Ud = cl.map_shared_rank(U, down);
            const float* Vd = cl.map_shared_rank(V, down);
            for (int i = tid; i < N; i += nthr) {           // 2 edge rows x N/2 pairs
                const int e = i / (N / 2), c = 2 * (i & (N / 2 - 1));
                const int r = e == 0 ? 1 : rp;
                if (e == 1 && rp == 1) continue;
                const int cl_ = (c + N - 1) & (N - 1), cr = (c + 2) & (N - 1);
                const int o = r * N;
                const float2 uU = r == 1 ? ld2(Uu + rp * N + c) : ld2(U + o - N + c);
                const float2 vU = r == 1 ? ld2(Vu + rp * N + c) : ld2(V + o - N + c);
                const float2 uD = r == rp ? ld2(Ud + N + c) : ld2(U + o + N + c);
                const float2 vD = r == rp ? ld2(Vd + N + c) : ld2(V + o + N + c);
                float2 un, vn;
                gs_update2(k, uU, ld2(U + o + c), uD, U[o + cl_], U[o + cr], vU, ld2(V + o + c), vD, V[o + cl_],
                           V[o + cr], &un, &vn);
                st2(Un + o + c, un);
                st2(Vn + o + c, vn);
            }
            if (tid < N) cluster_release();   // this thread wrote edge-row cells the neighbours read
        }
        __syncthreads();
        cluster_arrive_relaxed();
    }
    cluster_wait();
    const int fin = a.steps & 1;
    for (int i = tid; i < rp * N / 4; i += nthr) {
        reinterpret_cast<float4*>(uo + r0 * N)[i] = reinterpret_cast<const float4*>(sm + (2 * fin) * PL + N)[i];
        reinterpret_cast<float4*>(vo + r0 * N)[i] = reinterpret_cast<const float4*>(sm + (2 * fin + 1) * PL + N)[i];
    }
}

// ---- TMA bulk copies and mbarriers (inline PTX) ------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }

// Waits for phase `parity` of the mbarrier with an iteration limit: on timeout the
// error word is set and the wait gives up (the kernel still runs to completion, so
// every cluster barrier is still met; the host reports the error).
__device__ __forceinline__ void mbar_wait_bounded(uint64_t* bar, uint32_t parity, int* err) {
    uint32_t it = 0;
    while (!mbar_try_wait(bar, parity)) {
        if (++it == (1u << 22)) {
            atomicOr(err, 1);
            return;
        }
    }
}

// adjoint update of a column pair (transpose of gs_update2), with the gradient
// partial sums of gs_adj_update in packed form
// (any pairing of cells, full neighbour pairs; DRIFT as in gs_update2f)
template <int DRIFT = -1>
__device__ __forceinline__ void gs_adj_update2f(const GSCoef2& k, float2 aL, float2 aR, float2 aU, float2 aC, float2 aD,
                                                float2 bL, float2 bR, float2 bU, float2 bC, float2 bD, float2 uL,
                                                float2 uR, float2 uU, float2 uC, float2 uD, float2 vL, float2 vR,
                                                float2 vU, float2 vC, float2 vD, float2* an, float2* bn, float2 t[6]) {
    const float2 lap_a = fma2(k.m4, aC, add2(add2(aL, aR), add2(aU, aD)));
    const float2 lap_b = fma2(k.m4, bC, add2(add2(bL, bR), add2(bU, bD)));
    const float2 ba = sub2(bC, aC);
    float2 x = fma2(k.du, lap_a, mul2(k.mdtF, aC));
    float2 y = fma2(k.dv, lap_b, mul2(k.mdtFk, bC));
    if (DRIFT == 1 || (DRIFT < 0 && k.drift)) {
        x = fma2(k.hx, sub2(aR, aL), fma2(k.hy, sub2(aD, aU), x));
        y = fma2(k.hx, sub2(bR, bL), fma2(k.hy, sub2(bD, bU), y));
    }
    x = fma2(mul2(k.dt, mul2(vC, vC)), ba, x);
    y = fma2(mul2(k.two_dt, mul2(uC, vC)), ba, y);
    *an = add2(aC, x);
    *bn = add2(bC, y);
    const float2 lu = fma2(k.m4, uC, add2(add2(uL, uR), add2(uU, uD)));
    const float2 lv = fma2(k.m4, vC, add2(add2(vL, vR), add2(vU, vD)));
    t[0] = fma2(aC, sub2(k.one, uC), t[0]);
    t[1] = fma2(bC, vC, t[1]);
    t[2] = fma2(aC, lu, t[2]);
    t[3] = fma2(bC, lv, t[3]);
    t[4] = fma2(aC, sub2(uR, uL), fma2(bC, sub2(vR, vL), t[4]));
    t[5] = fma2(aC, sub2(uD, uU), fma2(bC, sub2(vD, vU), t[5]));
}

// The same adjoint update with the gradient partial sums moved onto the adjoint
// field by summation by parts over the periodic lattice, which needs the forward
// state only at the cells themselves:
//   sum a lap(u) = sum u lap(a),   sum a (uR - uL) = -sum u (aR - aL)  (and in y).
// t[2], t[3] as in gs_adj_update2f; t[4], t[5] hold the NEGATED drift sums.  The
// adjoint fields an, bn are the same bits as gs_adj_update2f's.
template <int DRIFT>
__device__ __forceinline__ void gs_adj_update2s(const GSCoef2& k, float2 aL, float2 aR, float2 aU, float2 aC, float2 aD,
                                                float2 bL, float2 bR, float2 bU, float2 bC, float2 bD, float2 uC,
                                                float2 vC, float2* an, float2* bn, float2 t[6]) {
    const float2 lap_a = fma2(k.m4, aC, add2(add2(aL, aR), add2(aU, aD)));
    const float2 lap_b = fma2(k.m4, bC, add2(add2(bL, bR), add2(bU, bD)));
    const float2 ba = sub2(bC, aC);
    float2 x = fma2(k.du, lap_a, mul2(k.mdtF, aC));
    float2 y = fma2(k.dv, lap_b, mul2(k.mdtFk, bC));
    const float2 dxa = sub2(aR, aL), dya = sub2(aD, aU), dxb = sub2(bR, bL), dyb = sub2(bD, bU);
    if (DRIFT == 1) {
        x = fma2(k.hx, dxa, fma2(k.hy, dya, x));
        y = fma2(k.hx, dxb, fma2(k.hy, dyb, y));
    }
    x = fma2(mul2(k.dt, mul2(vC, vC)), ba, x);
    y = fma2(mul2(k.two_dt, mul2(uC, vC)), ba, y);
    *an = add2(aC, x);
    *bn = add2(bC, y);
    t[0] = fma2(aC, sub2(k.one, uC), t[0]);
    t[1] = fma2(bC, vC, t[1]);
    t[2] = fma2(uC, lap_a, t[2]);
    t[3] = fma2(vC, lap_b, t[3]);
    t[4] = fma2(uC, dxa, fma2(vC, dxb, t[4]));
    t[5] = fma2(uC, dya, fma2(vC, dyb, t[5]));
}

__device__ __forceinline__ void gs_adj_update2(const GSCoef2& k, float2 aU, float2 aC, float2 aD, float aLs, float aRs,
                                               float2 bU, float2 bC, float2 bD, float bLs, float bRs, float2 uU,
                                               float2 uC, float2 uD, float uLs, float uRs, float2 vU, float2 vC,
                                               float2 vD, float vLs, float vRs, float2* an, float2* bn, float2 t[6]) {
    gs_adj_update2f(k, make_float2(aLs, aC.x), make_float2(aC.y, aRs), aU, aC, aD, make_float2(bLs, bC.x),
                    make_float2(bC.y, bRs), bU, bC, bD, make_float2(uLs, uC.x), make_float2(uC.y, uRs), uU, uC, uD,
                    make_float2(vLs, vC.x), make_float2(vC.y, vRs), vU, vC, vD, an, bn, t);
}

template <int N>
__global__ void __launch_bounds__(512, 1) k_gs_adjoint_x2(GSArgs<float> a, const float* __restrict__ states, int len,
                                                         const float* __restrict__ lu_in,
                                                         const float* __restrict__ lv_in, float* __restrict__ lu_out,
                                                         float* __restrict__ lv_out, double* __restrict__ grad,
                                                         int* __restrict__ err) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float* sm = reinterpret_cast<float*>(smem_raw);
    __shared__ double red[6][32];
    __shared__ __align__(8) uint64_t mbar[2];
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
    const GSCoef2 k(a);
    const int PL = (rp + 2) * N;
    float* S0 = sm + 4 * PL;                  // state buffers [2][field][rp + 2][N]
    const uint32_t row_bytes = N * sizeof(float);
    // states[j] rows r0-1 .. r0+rp (periodic) into state buffer b
    auto prefetch = [&](int j, int b) {
        fence_proxy_async();
        mbar_expect_tx(&mbar[b], 2 * (rp + 2) * row_bytes);
        for (int f = 0; f < 2; ++f) {
            const float* src = states + (size_t)(2 * j + f) * NN;
            float* dst = S0 + (2 * b + f) * PL;
            bulk_g2s(dst, src + ((r0 + N - 1) & (N - 1)) * N, row_bytes, &mbar[b]);
            bulk_g2s(dst + N, src + r0 * N, rp * row_bytes, &mbar[b]);
            bulk_g2s(dst + (rp + 1) * N, src + ((r0 + rp) & (N - 1)) * N, row_bytes, &mbar[b]);
        }
    };
    if (tid == 0) {
        mbar_init(&mbar[0], 1);
        mbar_init(&mbar[1], 1);
        fence_mbar_init();
    }
    for (int i = tid; i < rp * N / 4; i += nthr) {
        reinterpret_cast<float4*>(sm + N)[i] = reinterpret_cast<const float4*>(lu_in + r0 * N)[i];
        reinterpret_cast<float4*>(sm + PL + N)[i] = reinterpret_cast<const float4*>(lv_in + r0 * N)[i];
    }
    __syncthreads();
    if (tid == 0 && len > 0) prefetch(len - 1, 0);
    double g[6] = {0, 0, 0, 0, 0, 0};
    cluster_arrive();
    for (int j = len - 1, s = 0; j >= 0; --j, ++s) {
        const int cur = s & 1, sb = s & 1;
        const float* A = sm + (2 * cur) * PL;
        const float* B = A + PL;
        float* An = sm + (2 * (cur ^ 1)) * PL;
        float* Bn = An + PL;
        if (tid == 0 && j > 0) prefetch(j - 1, sb ^ 1);
        mbar_wait_bounded(&mbar[sb], (uint32_t)((s >> 1) & 1), err);
        const float* Us = S0 + (2 * sb) * PL;     // rows 0..rp+1 = global rows r0-1..r0+rp
        const float* Vs = Us + PL;
        float2 t[6] = {f2(0.f), f2(0.f), f2(0.f), f2(0.f), f2(0.f), f2(0.f)};
        if (ilo <= ihi) {
            for (int p = threadIdx.x; p < N / 2; p += BX) {
                const int c = 2 * p;
                const int cl_ = (c + N - 1) & (N - 1), cr = (c + 2) & (N - 1);
                float2 uU = ld2(Us + (ilo - 1) * N + c), vU = ld2(Vs + (ilo - 1) * N + c);
                float2 uC = ld2(Us + ilo * N + c), vC = ld2(Vs + ilo * N + c);
                float2 aU = ld2(A + (ilo - 1) * N + c), bU = ld2(B + (ilo - 1) * N + c);
                float2 aC = ld2(A + ilo * N + c), bC = ld2(B + ilo * N + c);
                for (int r = ilo; r <= ihi; ++r) {
                    const int o = r * N;
                    const float2 uD = ld2(Us + o + N + c), vD = ld2(Vs + o + N + c);
                    const float2 aD = ld2(A + o + N + c), bD = ld2(B + o + N + c);
                    float2 an, bn;
                    gs_adj_update2(k, aU, aC, aD, A[o + cl_], A[o + cr], bU, bC, bD, B[o + cl_], B[o + cr], uU, uC, uD,
                                   Us[o + cl_], Us[o + cr], vU, vC, vD, Vs[o + cl_], Vs[o + cr], &an, &bn, t);
                    st2(An + o + c, an);
                    st2(Bn + o + c, bn);
                    uU = uC; uC = uD; vU = vC; vC = vD;
                    aU = aC; aC = aD; bU = bC; bC = bD;
                }
            }
        }
        cluster_wait();
        {
            const float* Au = cl.map_shared_rank(A, up);
            const float* Bu = cl.map_shared_rank(B, up);
            const float* Ad = cl.map_shared_rank(A, down);
            const float* Bd = cl.map_shared_rank(B, down);
            for (int i = tid; i < N; i += nthr) {
                const int e = i / (N / 2), c = 2 * (i & (N / 2 - 1));
                const int r = e == 0 ? 1 : rp;
                if (e == 1 && rp == 1) continue;
                const int cl_ = (c + N - 1) & (N - 1), cr = (c + 2) & (N - 1);
                const int o = r * N;
                const float2 aU = r == 1 ? ld2(Au + rp * N + c) : ld2(A + o - N + c);
                const float2 bU = r == 1 ? ld2(Bu + rp * N + c) : ld2(B + o - N + c);
                const float2 aD = r == rp ? ld2(Ad + N + c) : ld2(A + o + N + c);
                const float2 bD = r == rp ? ld2(Bd + N + c) : ld2(B + o + N + c);
                float2 an, bn;
                gs_adj_update2(k, aU, ld2(A + o + c), aD, A[o + cl_], A[o + cr], bU, ld2(B + o + c), bD, B[o + cl_],
                               B[o + cr], ld2(Us + o - N + c), ld2(Us + o + c), ld2(Us + o + N + c), Us[o + cl_],
                               Us[o + cr], ld2(Vs + o - N + c), ld2(Vs + o + c), ld2(Vs + o + N + c), Vs[o + cl_],
                               Vs[o + cr], &an, &bn, t);
                st2(An + o + c, an);
                st2(Bn + o + c, bn);
            }
            if (tid < N) cluster_release();
        }
#pragma unroll
        for (int q = 0; q < 6; ++q) g[q] += (double)t[q].x + (double)t[q].y;
        __syncthreads();
        cluster_arrive_relaxed();
    }
    cluster_wait();
    const int fin = len & 1;
    for (int i = tid; i < rp * N / 4; i += nthr) {
        reinterpret_cast<float4*>(lu_out + r0 * N)[i] = reinterpret_cast<const float4*>(sm + (2 * fin) * PL + N)[i];
        reinterpret_cast<float4*>(lv_out + r0 * N)[i] =
            reinterpret_cast<const float4*>(sm + (2 * fin + 1) * PL + N)[i];
    }
    grad_reduce(g, (double)a.dt, grad, red, tid, nthr);
}
