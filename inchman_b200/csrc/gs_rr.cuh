// Register-resident float32 Gray-Scott forward kernel.
//
// The lattice is split over ONE 16-CTA thread-block cluster, and inside each CTA
// over its warps: warp g (g = CTA rank * WPC + warp) owns R = N / (16 WPC) whole
// rows, kept in registers for the entire solve.  A lane owns 2H = N / 32 adjacent
// columns, packed into H float2 pairs (c_j, c_{j+H}) so that every horizontal
// neighbour pair of a packed operation is again one of the lane's pairs, except at
// the two lane edges, which take one value each from the neighbouring lanes by
// warp shuffle (periodic in x through the lane wrap).
//
// The only data a warp needs from elsewhere are two halo rows: the last row of the
// warp above and the first row of the warp below (periodic in y across the
// cluster).  Each step a warp
//   1. waits on its own mbarrier for the two halo rows of the current state,
//   2. computes its first and last rows of the next state and sends them to the
//      two neighbouring warps (st.async into the neighbour CTA's shared memory
//      with a complete_tx signal on the neighbour's mbarrier, or st.shared plus an
//      mbarrier arrive when the neighbour is in the same CTA),
//   3. computes its interior rows while the sends travel.
// There is no block or cluster barrier inside the time loop: a warp waits only for
// its two neighbours.  Halo buffers and mbarriers are double-buffered by step
// parity; a producer can refill a buffer only after it received the consumer's
// rows of the following step, which the consumer computes from that buffer, so
// no buffer is overwritten before it has been read.
//
// Every wait is bounded; a wait that gives up sets g_gs_fwd_err and the CTA's
// output is written as NaN, so a failure cannot pass silently.
//
// Included from gray_scott.cu after gs_f32x2.cuh (uses GSArgs, GSCoef2,
// gs_update2f, smem_u32, mbar_init, fence_mbar_init, cluster_arrive/wait).

constexpr int kRRCluster = 16;
constexpr uint32_t kRRWaitLimit = 1u << 20;

__device__ int g_gs_fwd_err;

__device__ __forceinline__ uint32_t rr_ctarank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;\n" : "=r"(r));
    return r;
}
__device__ __forceinline__ uint32_t rr_mapa(uint32_t addr, uint32_t rank) {
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;\n" : "=r"(r) : "r"(addr), "r"(rank));
    return r;
}
__device__ __forceinline__ void rr_st_async(uint32_t addr, float4 v, uint32_t bar) {
    asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.v4.f32 [%0], {%1, %2, %3, %4}, [%5];\n" ::"r"(
                     addr),
                 "f"(v.x), "f"(v.y), "f"(v.z), "f"(v.w), "r"(bar)
                 : "memory");
}
__device__ __forceinline__ void rr_st_async(uint32_t addr, float2 v, uint32_t bar) {
    asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.v2.f32 [%0], {%1, %2}, [%3];\n" ::"r"(addr),
                 "f"(v.x), "f"(v.y), "r"(bar)
                 : "memory");
}
__device__ __forceinline__ void rr_st_local(uint32_t addr, float4 v) {
    asm volatile("st.shared.v4.f32 [%0], {%1, %2, %3, %4};\n" ::"r"(addr), "f"(v.x), "f"(v.y), "f"(v.z), "f"(v.w)
                 : "memory");
}
__device__ __forceinline__ void rr_st_local(uint32_t addr, float2 v) {
    asm volatile("st.shared.v2.f32 [%0], {%1, %2};\n" ::"r"(addr), "f"(v.x), "f"(v.y) : "memory");
}
__device__ __forceinline__ void rr_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.release.cta.shared::cta.b64 _, [%0];\n" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void rr_arm(uint32_t bar, uint32_t tx) {
    asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(tx)
                 : "memory");
}
__device__ __forceinline__ bool rr_test(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait: at most kRRWaitLimit polls (each try_wait may also suspend the
// warp for a short, hardware-defined time).  After the first wait of a CTA gave up, its later waits return at once,
// so a failure costs one wait limit, not one per step.
__device__ __forceinline__ void rr_wait(uint32_t bar, uint32_t parity, volatile int* failed) {
    if (*failed) return;
    uint32_t it = 0;
    while (!rr_test(bar, parity)) {
        if (++it == kRRWaitLimit) {
            *failed = 1;
            return;
        }
    }
}

// one lane's 2H columns [p, p + 2H) <-> its H pairs (c_j, c_{j+H})
template <int H>
__device__ __forceinline__ void rr_load(const float* __restrict__ p, float2 (&x)[H]) {
    if constexpr (H % 4 == 0) {
#pragma unroll
        for (int q = 0; q < H / 4; ++q) {
            const float4 a = reinterpret_cast<const float4*>(p)[q];
            const float4 b = reinterpret_cast<const float4*>(p + H)[q];
            x[4 * q] = make_float2(a.x, b.x);
            x[4 * q + 1] = make_float2(a.y, b.y);
            x[4 * q + 2] = make_float2(a.z, b.z);
            x[4 * q + 3] = make_float2(a.w, b.w);
        }
    } else if constexpr (H == 2) {
        const float2 a = reinterpret_cast<const float2*>(p)[0], b = reinterpret_cast<const float2*>(p + 2)[0];
        x[0] = make_float2(a.x, b.x);
        x[1] = make_float2(a.y, b.y);
    } else {
        x[0] = reinterpret_cast<const float2*>(p)[0];
    }
}
template <int H>
__device__ __forceinline__ void rr_store(float* __restrict__ p, const float2 (&x)[H]) {
    if constexpr (H % 4 == 0) {
#pragma unroll
        for (int q = 0; q < H / 4; ++q) {
            reinterpret_cast<float4*>(p)[q] = make_float4(x[4 * q].x, x[4 * q + 1].x, x[4 * q + 2].x, x[4 * q + 3].x);
            reinterpret_cast<float4*>(p + H)[q] =
                make_float4(x[4 * q].y, x[4 * q + 1].y, x[4 * q + 2].y, x[4 * q + 3].y);
        }
    } else if constexpr (H == 2) {
        reinterpret_cast<float2*>(p)[0] = make_float2(x[0].x, x[1].x);
        reinterpret_cast<float2*>(p + 2)[0] = make_float2(x[0].y, x[1].y);
    } else {
        reinterpret_cast<float2*>(p)[0] = x[0];
    }
}

// halo row of one field in shared memory: units of two pairs (one pair for H = 1),
// unit q of lane l at byte (q * 32 + l) * unit size, conflict-free for the warp
template <int H>
struct RRUnit {
    static constexpr int kCount = H >= 2 ? H / 2 : 1;
    static constexpr uint32_t kBytes = H >= 2 ? 16 : 8;
};

template <int H>
__device__ __forceinline__ void rr_read_halo(const unsigned char* base, int lane, float2 (&x)[H]) {
    if constexpr (H >= 2) {
#pragma unroll
        for (int q = 0; q < H / 2; ++q) {
            const float4 t = reinterpret_cast<const float4*>(base)[q * 32 + lane];
            x[2 * q] = make_float2(t.x, t.y);
            x[2 * q + 1] = make_float2(t.z, t.w);
        }
    } else {
        x[0] = reinterpret_cast<const float2*>(base)[lane];
    }
}

// sends one row (both fields) into the destination warp's halo slot: st.async with
// a complete_tx on the destination's mbarrier when it lives in another CTA, else
// st.shared and one mbarrier arrive per lane.  dst_u / dst_v / bar are addresses
// in the destination CTA's shared-memory layout.
template <int H>
__device__ __forceinline__ void rr_send(const float2 (&pu)[H], const float2 (&pv)[H], uint32_t dst_u, uint32_t dst_v,
                                        uint32_t bar, bool remote, uint32_t rank, int lane) {
    constexpr uint32_t UB = RRUnit<H>::kBytes;
    auto unit = [](const float2 (&p)[H], int q) {
        if constexpr (H >= 2) {
            return make_float4(p[2 * q].x, p[2 * q].y, p[2 * q + 1].x, p[2 * q + 1].y);
        } else {
            return p[0];
        }
    };
    if (remote) {
        const uint32_t ru = rr_mapa(dst_u, rank), rv = rr_mapa(dst_v, rank), rb = rr_mapa(bar, rank);
#pragma unroll
        for (int q = 0; q < RRUnit<H>::kCount; ++q) {
            const uint32_t off = (uint32_t)(q * 32 + lane) * UB;
            rr_st_async(ru + off, unit(pu, q), rb);
            rr_st_async(rv + off, unit(pv, q), rb);
        }
    } else {
#pragma unroll
        for (int q = 0; q < RRUnit<H>::kCount; ++q) {
            const uint32_t off = (uint32_t)(q * 32 + lane) * UB;
            rr_st_local(dst_u + off, unit(pu, q));
            rr_st_local(dst_v + off, unit(pv, q));
        }
        rr_arrive(bar);
    }
}

// next state of one row from the rows above (U), at (C) and below (D)
template <int H, int DRIFT>
__device__ __forceinline__ void rr_row(const GSCoef2& k, const float2 (&uU)[H], const float2 (&uC)[H],
                                       const float2 (&uD)[H], const float2 (&vU)[H], const float2 (&vC)[H],
                                       const float2 (&vD)[H], float2 (&un)[H], float2 (&vn)[H], int lane) {
    const int lft = (lane + 31) & 31, rgt = (lane + 1) & 31;
    const float ul = __shfl_sync(0xffffffffu, uC[H - 1].y, lft), ur = __shfl_sync(0xffffffffu, uC[0].x, rgt);
    const float vl = __shfl_sync(0xffffffffu, vC[H - 1].y, lft), vr = __shfl_sync(0xffffffffu, vC[0].x, rgt);
#pragma unroll
    for (int j = 0; j < H; ++j) {
        const float2 uL = j == 0 ? make_float2(ul, uC[H - 1].x) : uC[j == 0 ? 0 : j - 1];
        const float2 uR = j == H - 1 ? make_float2(uC[0].y, ur) : uC[j == H - 1 ? 0 : j + 1];
        const float2 vL = j == 0 ? make_float2(vl, vC[H - 1].x) : vC[j == 0 ? 0 : j - 1];
        const float2 vR = j == H - 1 ? make_float2(vC[0].y, vr) : vC[j == H - 1 ? 0 : j + 1];
        gs_update2f<DRIFT>(k, uL, uR, uU[j], uC[j], uD[j], vL, vR, vU[j], vC[j], vD[j], &un[j], &vn[j]);
    }
}

template <int N, int WPC>
struct RRShape {
    static constexpr int R = N / (kRRCluster * WPC);   // rows per warp
    static constexpr int H = N / 64;                    // column pairs per lane
    static constexpr uint32_t kRow = 4u * N;            // bytes of one halo row of one field
    // [warp][parity][side above/below][field u/v] halo rows, then [warp][parity]
    // mbarriers, then the CTA's failure flag
    static constexpr uint32_t kHalo = (uint32_t)WPC * 8u * kRow;
    static constexpr uint32_t kSmem = kHalo + (uint32_t)WPC * 16u + 16u;
    static_assert(kSmem <= 227u * 1024u, "forward shared memory exceeds a B200 CTA's");
    static_assert(R >= 1 && R * kRRCluster * WPC == N && H >= 1 && 64 * H == N, "lattice split");
};

template <int N, int WPC>
struct RRCtx {
    using S = RRShape<N, WPC>;
    uint32_t sbase;
    const unsigned char* smem;
    int lane, w;
    uint32_t up_rank, dn_rank;
    int up_w, dn_w;
    bool up_remote, dn_remote;
    uint32_t tx;             // bytes the producers in other CTAs deliver per phase
    volatile int* failed;
    __device__ __forceinline__ uint32_t slot(int ww, int par, int side, int f) const {
        return sbase + (uint32_t)(((ww * 2 + par) * 2 + side) * 2 + f) * S::kRow;
    }
    __device__ __forceinline__ uint32_t bar(int ww, int par) const { return sbase + S::kHalo + (uint32_t)(ww * 2 + par) * 8u; }
};

// one step X -> Y of the warp's rows in registers (s: the step index of X; send:
// whether Y's edge rows go out, i.e. not after the last step).  The edge rows are
// computed and sent first; the interior rows are computed while the sends travel.
template <int N, int WPC, int DRIFT>
__device__ __forceinline__ void rr_step(const RRCtx<N, WPC>& c, const GSCoef2& k,
                                        const float2 (&xu)[RRShape<N, WPC>::R][RRShape<N, WPC>::H],
                                        const float2 (&xv)[RRShape<N, WPC>::R][RRShape<N, WPC>::H],
                                        float2 (&yu)[RRShape<N, WPC>::R][RRShape<N, WPC>::H],
                                        float2 (&yv)[RRShape<N, WPC>::R][RRShape<N, WPC>::H], int s, bool send) {
    constexpr int R = RRShape<N, WPC>::R, H = RRShape<N, WPC>::H;
    const int par = s & 1;
    rr_wait(c.bar(c.w, par), (uint32_t)(s >> 1) & 1u, c.failed);
    __syncwarp();
    if (c.lane == 0) rr_arm(c.bar(c.w, par), c.tx);   // the phase of step s + 2
    float2 au[H], av[H], bu[H], bv[H];
    rr_read_halo<H>(c.smem + (c.slot(c.w, par, 0, 0) - c.sbase), c.lane, au);
    rr_read_halo<H>(c.smem + (c.slot(c.w, par, 0, 1) - c.sbase), c.lane, av);
    rr_read_halo<H>(c.smem + (c.slot(c.w, par, 1, 0) - c.sbase), c.lane, bu);
    rr_read_halo<H>(c.smem + (c.slot(c.w, par, 1, 1) - c.sbase), c.lane, bv);
    if constexpr (R == 1) {
        rr_row<H, DRIFT>(k, au, xu[0], bu, av, xv[0], bv, yu[0], yv[0], c.lane);
    } else {
        rr_row<H, DRIFT>(k, au, xu[0], xu[1], av, xv[0], xv[1], yu[0], yv[0], c.lane);
        rr_row<H, DRIFT>(k, xu[R - 2], xu[R - 1], bu, xv[R - 2], xv[R - 1], bv, yu[R - 1], yv[R - 1], c.lane);
    }
    if (send) {
        const int np = par ^ 1;
        // first row -> the warp above (its lower halo), last row -> the warp below (its upper halo)
        rr_send<H>(yu[0], yv[0], c.slot(c.up_w, np, 1, 0), c.slot(c.up_w, np, 1, 1), c.bar(c.up_w, np), c.up_remote,
                   c.up_rank, c.lane);
        rr_send<H>(yu[R - 1], yv[R - 1], c.slot(c.dn_w, np, 0, 0), c.slot(c.dn_w, np, 0, 1), c.bar(c.dn_w, np),
                   c.dn_remote, c.dn_rank, c.lane);
    }
#pragma unroll
    for (int r = 1; r < R - 1; ++r)
        rr_row<H, DRIFT>(k, xu[r - 1], xu[r], xu[r + 1], xv[r - 1], xv[r], xv[r + 1], yu[r], yv[r], c.lane);
}

template <int N, int WPC, int DRIFT>
__global__ void __launch_bounds__(32 * WPC, 1)
    k_gs_forward_rr(GSArgs<float> a, const float* __restrict__ u0, const float* __restrict__ v0,
                    float* __restrict__ uo, float* __restrict__ vo, float* __restrict__ trace, int trace_every,
                    const GSArgs<float>* __restrict__ batch_args) {
    using S = RRShape<N, WPC>;
    constexpr int R = S::R, H = S::H;
    constexpr int NN = N * N;
    // a batched launch runs one lattice per cluster: member m = cluster index, with
    // its own state slice and parameters (trace is single-lattice only)
    const int member = (int)blockIdx.x / kRRCluster;
    if (batch_args) {
        const size_t moff = (size_t)member * NN;
        u0 += moff; v0 += moff; uo += moff; vo += moff;
        a = batch_args[member];
        trace = nullptr;
    }
    extern __shared__ __align__(16) unsigned char smem_raw[];
    RRCtx<N, WPC> c;
    c.smem = smem_raw;
    c.sbase = smem_u32(smem_raw);
    c.lane = threadIdx.x & 31;
    c.w = threadIdx.x >> 5;
    const uint32_t rank = rr_ctarank();
    c.up_remote = c.w == 0;
    c.dn_remote = c.w == WPC - 1;
    c.up_rank = c.up_remote ? (rank + kRRCluster - 1) % kRRCluster : rank;
    c.dn_rank = c.dn_remote ? (rank + 1) % kRRCluster : rank;
    c.up_w = c.up_remote ? WPC - 1 : c.w - 1;
    c.dn_w = c.dn_remote ? 0 : c.w + 1;
    c.failed = reinterpret_cast<volatile int*>(smem_raw + S::kHalo + WPC * 16);
    const int nremote = (int)c.up_remote + (int)c.dn_remote;
    c.tx = (uint32_t)nremote * 2u * S::kRow;
    const int row0 = ((int)rank * WPC + c.w) * R;
    const int col0 = c.lane * 2 * H;
    const GSCoef2 k(a);

    if (c.lane == 0) {
        // arrivals per phase: the own arm + 32 lanes of every producer warp in this CTA
        mbar_init(reinterpret_cast<uint64_t*>(smem_raw + (c.bar(c.w, 0) - c.sbase)), 1 + 32 * (2 - nremote));
        mbar_init(reinterpret_cast<uint64_t*>(smem_raw + (c.bar(c.w, 1) - c.sbase)), 1 + 32 * (2 - nremote));
        fence_mbar_init();
    }
    if (threadIdx.x == 0) *c.failed = 0;
    float2 xu[R][H], xv[R][H], yu[R][H], yv[R][H];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        rr_load<H>(u0 + (size_t)(row0 + r) * N + col0, xu[r]);
        rr_load<H>(v0 + (size_t)(row0 + r) * N + col0, xv[r]);
    }
    __syncthreads();
    cluster_arrive();     // every CTA's mbarriers exist before anyone sends
    cluster_wait();
    const int steps = a.steps;
    const int every = trace_every > 0 ? trace_every : 1;
    if (steps > 0) {
        if (c.lane == 0) {
            rr_arm(c.bar(c.w, 0), c.tx);
            rr_arm(c.bar(c.w, 1), c.tx);
        }
        rr_send<H>(xu[0], xv[0], c.slot(c.up_w, 0, 1, 0), c.slot(c.up_w, 0, 1, 1), c.bar(c.up_w, 0), c.up_remote,
                   c.up_rank, c.lane);
        rr_send<H>(xu[R - 1], xv[R - 1], c.slot(c.dn_w, 0, 0, 0), c.slot(c.dn_w, 0, 0, 1), c.bar(c.dn_w, 0),
                   c.dn_remote, c.dn_rank, c.lane);
    }
    auto put_trace = [&](int s, const float2 (&pu)[R][H], const float2 (&pv)[R][H]) {
        if (trace != nullptr && s % every == 0) {
            float* du = trace + (size_t)(2 * (s / every)) * NN;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                rr_store<H>(du + (size_t)(row0 + r) * N + col0, pu[r]);
                rr_store<H>(du + NN + (size_t)(row0 + r) * N + col0, pv[r]);
            }
        }
    };
    int s = 0;
    for (; s + 2 <= steps; s += 2) {      // two steps per iteration: X -> Y -> X without copies
        put_trace(s, xu, xv);
        rr_step<N, WPC, DRIFT>(c, k, xu, xv, yu, yv, s, true);
        put_trace(s + 1, yu, yv);
        rr_step<N, WPC, DRIFT>(c, k, yu, yv, xu, xv, s + 1, s + 2 < steps);
    }
    const bool odd = s < steps;
    if (odd) {
        put_trace(s, xu, xv);
        rr_step<N, WPC, DRIFT>(c, k, xu, xv, yu, yv, s, false);
    }
    __syncthreads();
    cluster_arrive();     // no CTA leaves while a neighbour may still address its shared memory
    cluster_wait();
    const bool bad = *c.failed != 0;
    if (bad && threadIdx.x == 0) atomicOr(&g_gs_fwd_err, 1);
    const float nan = __int_as_float(0x7fc00000);
#pragma unroll
    for (int r = 0; r < R; ++r) {
        float2 pu[H], pv[H];
#pragma unroll
        for (int j = 0; j < H; ++j) {
            pu[j] = bad ? make_float2(nan, nan) : (odd ? yu[r][j] : xu[r][j]);
            pv[j] = bad ? make_float2(nan, nan) : (odd ? yv[r][j] : xv[r][j]);
        }
        rr_store<H>(uo + (size_t)(row0 + r) * N + col0, pu);
        rr_store<H>(vo + (size_t)(row0 + r) * N + col0, pv);
    }
}

// ---- register-resident adjoint -----------------------------------------------------
// The transposed steps of a segment, last to first, with the adjoint fields
// (lambda_u, lambda_v) in registers and exchanged between warps exactly like the
// forward state.  The stored forward states of the segment stream through shared
// memory: lane 0 of warp 0 issues TMA bulk copies (cp.async.bulk, completion on a
// "full" mbarrier) of the CTA's rows two steps ahead into a ring of four buffers;
// every warp releases a buffer on an "empty" mbarrier when it is done with it, and
// a buffer is refilled only after all warps released it.  The per-cell update is
// gs_adj_update2s: the adjoint fields are bit-identical to the shared-memory
// adjoint kernel's, and the parameter-gradient sums, taken by parts over the
// periodic lattice, need the forward state only at the cell itself (so no state
// halo rows).  The partial sums are formed per lane and step in float and summed
// in double.

template <int N, int WPC>
struct RRAdjShape {
    using F = RRShape<N, WPC>;
    static constexpr int R = F::R, H = F::H;
    static constexpr int RC = WPC * R;                      // rows per CTA
    static constexpr int NB = 4;                            // state buffers in the ring
    static constexpr int kAhead = 2;                        // steps issued ahead
    static constexpr uint32_t kPipe = F::kHalo + (uint32_t)WPC * 16u;   // full[NB], empty[NB]
    static constexpr uint32_t kFlag = kPipe + 16u * NB;
    static constexpr uint32_t kState = (kFlag + 16u + 127u) / 128u * 128u;   // [buf][field][RC][N]
    static constexpr uint32_t kPlane = (uint32_t)RC * 4u * N;
    static constexpr uint32_t kSmem = kState + 2u * NB * kPlane;
    static_assert(kSmem <= 227u * 1024u, "adjoint shared memory exceeds a B200 CTA's");
};

template <int H, int DRIFT>
__device__ __forceinline__ void rr_adj_row(const GSCoef2& k, const float2 (&aU)[H], const float2 (&aC)[H],
                                           const float2 (&aD)[H], const float2 (&bU)[H], const float2 (&bC)[H],
                                           const float2 (&bD)[H], const float2 (&uC)[H], const float2 (&vC)[H],
                                           float2 (&an)[H], float2 (&bn)[H], float2 t[6], int lane) {
    const int lft = (lane + 31) & 31, rgt = (lane + 1) & 31;
    const float al = __shfl_sync(0xffffffffu, aC[H - 1].y, lft), ar = __shfl_sync(0xffffffffu, aC[0].x, rgt);
    const float bl = __shfl_sync(0xffffffffu, bC[H - 1].y, lft), br = __shfl_sync(0xffffffffu, bC[0].x, rgt);
#pragma unroll
    for (int j = 0; j < H; ++j) {
        const int jl = j == 0 ? 0 : j - 1, jr = j == H - 1 ? 0 : j + 1;
        const float2 aL = j == 0 ? make_float2(al, aC[H - 1].x) : aC[jl];
        const float2 aR = j == H - 1 ? make_float2(aC[0].y, ar) : aC[jr];
        const float2 bL = j == 0 ? make_float2(bl, bC[H - 1].x) : bC[jl];
        const float2 bR = j == H - 1 ? make_float2(bC[0].y, br) : bC[jr];
        gs_adj_update2s<DRIFT>(k, aL, aR, aU[j], aC[j], aD[j], bL, bR, bU[j], bC[j], bD[j], uC[j], vC[j], &an[j],
                               &bn[j], t);
    }
}

// issues the TMA copies of the forward state of adjoint step q (stored state
// len - 1 - q) into ring buffer q % NB, after all warps released that buffer's
// previous use (step q - NB); one thread
template <int N, int WPC>
__device__ __forceinline__ void rr_adj_issue(const RRCtx<N, WPC>& c, const float* __restrict__ states, int len, int q,
                                             int rc0) {
    using S = RRAdjShape<N, WPC>;
    constexpr int NN = N * N;
    const int b = q % S::NB, j = len - 1 - q;
    uint64_t* full = reinterpret_cast<uint64_t*>(const_cast<unsigned char*>(c.smem) + S::kPipe) + b;
    if (q >= S::NB) rr_wait(c.sbase + S::kPipe + 8u * (S::NB + b), (uint32_t)((q - S::NB) / S::NB) & 1u, c.failed);
    fence_proxy_async();
    mbar_expect_tx(full, 2u * S::kPlane);
    for (int f = 0; f < 2; ++f) {
        const float* src = states + (size_t)(2 * j + f) * NN + (size_t)rc0 * N;
        float* dst = reinterpret_cast<float*>(const_cast<unsigned char*>(c.smem) + S::kState +
                                              (uint32_t)(2 * b + f) * S::kPlane);
        bulk_g2s(dst, src, S::kPlane, full);
    }
}

// one transposed step X -> Y of the warp's adjoint rows; the forward state of the
// step is buffer s % NB of the state ring
template <int N, int WPC, int DRIFT>
__device__ __forceinline__ void rr_adj_step(const RRCtx<N, WPC>& c, const GSCoef2& k,
                                            const float2 (&xa)[RRShape<N, WPC>::R][RRShape<N, WPC>::H],
                                            const float2 (&xb)[RRShape<N, WPC>::R][RRShape<N, WPC>::H],
                                            float2 (&ya)[RRShape<N, WPC>::R][RRShape<N, WPC>::H],
                                            float2 (&yb)[RRShape<N, WPC>::R][RRShape<N, WPC>::H], int s, bool send,
                                            float2 t[6]) {
    using S = RRAdjShape<N, WPC>;
    constexpr int R = S::R, H = S::H;
    const int par = s & 1, sb = s % S::NB;
    const uint32_t full = c.sbase + S::kPipe + 8u * sb;
    const uint32_t empty = c.sbase + S::kPipe + 8u * (S::NB + sb);
    rr_wait(full, (uint32_t)(s / S::NB) & 1u, c.failed);        // the forward state of this step
    rr_wait(c.bar(c.w, par), (uint32_t)(s >> 1) & 1u, c.failed);   // the adjoint halo rows
    __syncwarp();
    if (c.lane == 0) rr_arm(c.bar(c.w, par), c.tx);
    float2 ha[H], hb[H], la[H], lb[H];
    rr_read_halo<H>(c.smem + (c.slot(c.w, par, 0, 0) - c.sbase), c.lane, ha);
    rr_read_halo<H>(c.smem + (c.slot(c.w, par, 0, 1) - c.sbase), c.lane, hb);
    rr_read_halo<H>(c.smem + (c.slot(c.w, par, 1, 0) - c.sbase), c.lane, la);
    rr_read_halo<H>(c.smem + (c.slot(c.w, par, 1, 1) - c.sbase), c.lane, lb);
    // the forward state at the warp's rows (shared-memory rows w R .. w R + R - 1)
    const float* Us = reinterpret_cast<const float*>(c.smem + S::kState + (uint32_t)(2 * sb) * S::kPlane);
    const float* Vs = reinterpret_cast<const float*>(c.smem + S::kState + (uint32_t)(2 * sb + 1) * S::kPlane);
    const int col0 = c.lane * 2 * H;
    float2 su[R][H], sv[R][H];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        rr_load<H>(Us + (c.w * R + r) * N + col0, su[r]);
        rr_load<H>(Vs + (c.w * R + r) * N + col0, sv[r]);
    }
    if constexpr (R == 1) {
        rr_adj_row<H, DRIFT>(k, ha, xa[0], la, hb, xb[0], lb, su[0], sv[0], ya[0], yb[0], t, c.lane);
    } else {
        rr_adj_row<H, DRIFT>(k, ha, xa[0], xa[1], hb, xb[0], xb[1], su[0], sv[0], ya[0], yb[0], t, c.lane);
        rr_adj_row<H, DRIFT>(k, xa[R - 2], xa[R - 1], la, xb[R - 2], xb[R - 1], lb, su[R - 1], sv[R - 1], ya[R - 1],
                             yb[R - 1], t, c.lane);
    }
    if (send) {
        const int np = par ^ 1;
        rr_send<H>(ya[0], yb[0], c.slot(c.up_w, np, 1, 0), c.slot(c.up_w, np, 1, 1), c.bar(c.up_w, np), c.up_remote,
                   c.up_rank, c.lane);
        rr_send<H>(ya[R - 1], yb[R - 1], c.slot(c.dn_w, np, 0, 0), c.slot(c.dn_w, np, 0, 1), c.bar(c.dn_w, np),
                   c.dn_remote, c.dn_rank, c.lane);
    }
#pragma unroll
    for (int r = 1; r < R - 1; ++r)
        rr_adj_row<H, DRIFT>(k, xa[r - 1], xa[r], xa[r + 1], xb[r - 1], xb[r], xb[r + 1], su[r], sv[r], ya[r], yb[r], t,
                             c.lane);
    __syncwarp();
    if (c.lane == 0) rr_arrive(empty);                       // this warp is done with the state buffer
}

template <int N, int WPC, int DRIFT>
__global__ void __launch_bounds__(32 * WPC, 1)
    k_gs_adjoint_rr(GSArgs<float> a, const float* __restrict__ states, int len, const float* __restrict__ lu_in,
                    const float* __restrict__ lv_in, float* __restrict__ lu_out, float* __restrict__ lv_out,
                    double* __restrict__ grad, int* __restrict__ err) {
    using S = RRAdjShape<N, WPC>;
    constexpr int R = S::R, H = S::H, RC = S::RC;
    constexpr int NN = N * N;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ double red[6][32];
    RRCtx<N, WPC> c;
    c.smem = smem_raw;
    c.sbase = smem_u32(smem_raw);
    c.lane = threadIdx.x & 31;
    c.w = threadIdx.x >> 5;
    const uint32_t rank = rr_ctarank();
    c.up_remote = c.w == 0;
    c.dn_remote = c.w == WPC - 1;
    c.up_rank = c.up_remote ? (rank + kRRCluster - 1) % kRRCluster : rank;
    c.dn_rank = c.dn_remote ? (rank + 1) % kRRCluster : rank;
    c.up_w = c.up_remote ? WPC - 1 : c.w - 1;
    c.dn_w = c.dn_remote ? 0 : c.w + 1;
    c.failed = reinterpret_cast<volatile int*>(smem_raw + S::kFlag);
    const int nremote = (int)c.up_remote + (int)c.dn_remote;
    c.tx = (uint32_t)nremote * 2u * RRShape<N, WPC>::kRow;
    uint64_t* pipe = reinterpret_cast<uint64_t*>(smem_raw + S::kPipe);   // full[0..NB-1], empty[0..NB-1]
    const int rc0 = (int)rank * RC;
    const int row0 = rc0 + c.w * R;
    const int col0 = c.lane * 2 * H;
    const GSCoef2 k(a);

    const bool issuer = threadIdx.x == 0;
    if (issuer) {
        for (int b = 0; b < S::NB; ++b) {
            mbar_init(&pipe[b], 1);
            mbar_init(&pipe[S::NB + b], WPC);
        }
        *c.failed = 0;
        fence_mbar_init();
    }
    if (c.lane == 0) {
        mbar_init(reinterpret_cast<uint64_t*>(smem_raw + (c.bar(c.w, 0) - c.sbase)), 1 + 32 * (2 - nremote));
        mbar_init(reinterpret_cast<uint64_t*>(smem_raw + (c.bar(c.w, 1) - c.sbase)), 1 + 32 * (2 - nremote));
        fence_mbar_init();
    }
    float2 xa[R][H], xb[R][H], ya[R][H], yb[R][H];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        rr_load<H>(lu_in + (size_t)(row0 + r) * N + col0, xa[r]);
        rr_load<H>(lv_in + (size_t)(row0 + r) * N + col0, xb[r]);
    }
    __syncthreads();
    cluster_arrive();     // every CTA's mbarriers exist before anyone sends
    cluster_wait();
    double g[6] = {0, 0, 0, 0, 0, 0};
    if (issuer)
        for (int q = 0; q < S::kAhead && q < len; ++q) rr_adj_issue<N, WPC>(c, states, len, q, rc0);
    if (len > 0) {
        if (c.lane == 0) {
            rr_arm(c.bar(c.w, 0), c.tx);
            rr_arm(c.bar(c.w, 1), c.tx);
        }
        rr_send<H>(xa[0], xb[0], c.slot(c.up_w, 0, 1, 0), c.slot(c.up_w, 0, 1, 1), c.bar(c.up_w, 0), c.up_remote,
                   c.up_rank, c.lane);
        rr_send<H>(xa[R - 1], xb[R - 1], c.slot(c.dn_w, 0, 0, 0), c.slot(c.dn_w, 0, 0, 1), c.bar(c.dn_w, 0),
                   c.dn_remote, c.dn_rank, c.lane);
    }
    // gradient partial sums: float over the two steps of an iteration, then double
    auto flush = [&](float2 (&t)[6]) {
#pragma unroll
        for (int q = 0; q < 6; ++q) {
            g[q] += (double)t[q].x + (double)t[q].y;
            t[q] = f2(0.f);
        }
    };
    float2 t[6] = {f2(0.f), f2(0.f), f2(0.f), f2(0.f), f2(0.f), f2(0.f)};
    int s = 0;
    for (; s + 2 <= len; s += 2) {
        if (issuer && s + S::kAhead < len) rr_adj_issue<N, WPC>(c, states, len, s + S::kAhead, rc0);
        rr_adj_step<N, WPC, DRIFT>(c, k, xa, xb, ya, yb, s, true, t);
        if (issuer && s + 1 + S::kAhead < len) rr_adj_issue<N, WPC>(c, states, len, s + 1 + S::kAhead, rc0);
        rr_adj_step<N, WPC, DRIFT>(c, k, ya, yb, xa, xb, s + 1, s + 2 < len, t);
        flush(t);
    }
    const bool odd = s < len;
    if (odd) {
        rr_adj_step<N, WPC, DRIFT>(c, k, xa, xb, ya, yb, s, false, t);
        flush(t);
    }
    g[4] = -g[4];      // gs_adj_update2s accumulates the drift sums negated
    g[5] = -g[5];
    __syncthreads();
    cluster_arrive();     // no CTA leaves while a neighbour may still address its shared memory
    cluster_wait();
    const bool bad = *c.failed != 0;
    if (bad && threadIdx.x == 0) atomicOr(err, 1);
    const float nan = __int_as_float(0x7fc00000);
#pragma unroll
    for (int r = 0; r < R; ++r) {
        float2 pa[H], pb[H];
#pragma unroll
        for (int j = 0; j < H; ++j) {
            pa[j] = bad ? make_float2(nan, nan) : (odd ? ya[r][j] : xa[r][j]);
            pb[j] = bad ? make_float2(nan, nan) : (odd ? yb[r][j] : xb[r][j]);
        }
        rr_store<H>(lu_out + (size_t)(row0 + r) * N + col0, pa);
        rr_store<H>(lv_out + (size_t)(row0 + r) * N + col0, pb);
    }
    grad_reduce(g, (double)a.dt, grad, red, (int)threadIdx.x, (int)blockDim.x);
}
