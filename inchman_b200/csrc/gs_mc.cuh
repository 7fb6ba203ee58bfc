// Register-resident float32 Gray-Scott forward kernel over C thread-block clusters.
//
// The single-cluster kernel (gs_rr.cuh) runs one lattice on 16 SMs; its step time is
// the arithmetic of 16 rows per SM plus one neighbour hop.  Here the lattice's N rows
// are cut into C bands of B = N / C rows, one band per 16-CTA cluster, so each SM
// holds a few rows (one per warp) and the arithmetic per step shrinks C-fold.
//
// Clusters cannot exchange rows through distributed shared memory, so each cluster
// also keeps G ghost rows on each side of its band (L = B + 2G rows per cluster, one
// per warp, WPC = L / 16 warps per CTA) and runs exactly the single-cluster kernel's
// ring inside the cluster: every step a warp waits for its two neighbours' rows,
// computes its row and sends it to them.  The ring's two ends (the outermost ghost
// rows) have no true neighbour, so a ghost row's value goes stale one row per step
// from the outside in; after G steps every ghost row is stale while the band rows,
// at least G rows from the ring's ends, are still exact.  At every state m * G the
// clusters swap rows through global memory: the G first and G last band rows of each
// cluster are written to an exchange buffer, every value packed with the block number
// m in one 64-bit word, and the warps that own the ghost rows poll the neighbouring
// clusters' words until all of them carry m, then send the fresh rows on.  A packed
// word is written by one single-copy atomic store, so neither side needs a flag or a
// fence: one trip through L2 instead of three (0.587 against 0.624 us per step with a
// release/acquire flag per lane at 8 ghost rows).  Every row of the band is therefore
// computed from exactly the values the single-cluster kernel uses: the result is
// bit-identical to it.
//
// The exchange buffer is double-buffered by the parity of m.  A cluster writes the
// block m + 2 buffer only after its ghost rows were refreshed at state (m + 1) G from
// rows its neighbour computed after reading block m, so no buffer is overwritten
// before it has been read; a word still holding block m - 2 fails the check.  The host
// clears the buffer on the launching stream before every launch (a captured graph
// replays that clear too), so no word of an earlier launch can carry m.  Every wait is
// bounded; a wait that gives up marks the CTA failed and its rows are written as NaN.
//
// All C clusters must be resident at once; the host checks that with
// cudaOccupancyMaxActiveClusters (shared memory is padded so one CTA holds one SM)
// and otherwise runs the single-cluster kernel.
//
// Included from gray_scott.cu after gs_rr.cuh.

constexpr uint32_t kMCSwapWaitLimit = 1u << 22;

template <int N, int C, int G, int WPC>
struct MCShape {
    static constexpr int B = N / C;                    // band rows per cluster
    static constexpr int L = B + 2 * G;                // rows per cluster (one per warp)
    static constexpr int H = N / 64;                   // column pairs per lane
    static constexpr uint32_t kRow = 4u * N;           // bytes of one halo row of one field
    static constexpr uint32_t kHalo = (uint32_t)WPC * 8u * kRow;
    static constexpr uint32_t kUsed = kHalo + (uint32_t)WPC * 16u + 16u;
    // at least 120 KB, so that no SM holds two CTAs (the steps are latency-bound: two
    // rows' arithmetic on one SM would lengthen every step)
    static constexpr uint32_t kSmem = kUsed > 120u * 1024u ? kUsed : 120u * 1024u;
    // exchange buffer: [parity][cluster][side][g] rows of 64-bit words (value bits, block
    // number), unit q (two words) of lane l at word (q * 32 + l) * 2; 4H words per lane
    static constexpr size_t kRowWords = (size_t)32 * 4 * H;
    static constexpr size_t kXWords = (size_t)2 * C * 2 * G * kRowWords;
    static_assert(N % C == 0 && C >= 2, "bands");
    static_assert(L == kRRCluster * WPC, "one row per warp");
    static_assert(B >= 2 * G && G >= 1, "band rows at least G rows from the ring's ends");
    static_assert(kSmem <= 227u * 1024u, "shared memory of a B200 CTA");
    static_assert(64 * H == N, "lane layout");
};

template <int N, int C, int G, int WPC>
struct MCCtx {
    using S = MCShape<N, C, G, WPC>;
    uint32_t sbase;
    const unsigned char* smem;
    int lane, w;
    uint32_t up_rank, dn_rank;
    int up_w, dn_w;
    bool up_remote, dn_remote;
    uint32_t tx;             // bytes the producers in other CTAs deliver per phase
    volatile int* failed;
    // exchange roles of this warp's row: source of a neighbour's ghost row, or ghost row
    uint64_t* src_row;          // where this row goes at a swap, or nullptr
    const uint64_t* ghost_row;  // where this row comes from at a swap, or nullptr
    size_t parity_stride;       // words between the two parities of the exchange buffer
    __device__ __forceinline__ uint32_t slot(int ww, int par, int side, int f) const {
        return sbase + (uint32_t)(((ww * 2 + par) * 2 + side) * 2 + f) * S::kRow;
    }
    __device__ __forceinline__ uint32_t bar(int ww, int par) const { return sbase + S::kHalo + (uint32_t)(ww * 2 + par) * 8u; }
};

// the swap at state m * G of a warp's freshly computed row y (see the file comment):
// every value travels packed with the block number m in one 64-bit word (a single-copy
// atomic store), so the reader needs no flag and no fence: it polls the words until
// all of them carry m
__device__ __forceinline__ uint64_t mc_pack(float v, int m) {
    return ((uint64_t)(uint32_t)m << 32) | (uint64_t)__float_as_uint(v);
}
template <int N, int C, int G, int WPC>
__device__ __forceinline__ void mc_swap(const MCCtx<N, C, G, WPC>& c, float2 (&yu)[N / 64], float2 (&yv)[N / 64],
                                        int m) {
    constexpr int H = N / 64;
    const size_t poff = (size_t)(m & 1) * c.parity_stride;
    if (c.src_row) {
        uint64_t* d = c.src_row + poff;
#pragma unroll
        for (int j = 0; j < H; ++j) {
            const ulonglong2 a = make_ulonglong2(mc_pack(yu[j].x, m), mc_pack(yu[j].y, m));
            const ulonglong2 b = make_ulonglong2(mc_pack(yv[j].x, m), mc_pack(yv[j].y, m));
            asm volatile("st.global.v2.u64 [%0], {%1, %2};\n" ::"l"(d + (size_t)(j * 32 + c.lane) * 2), "l"(a.x), "l"(a.y)
                         : "memory");
            asm volatile("st.global.v2.u64 [%0], {%1, %2};\n" ::"l"(d + (size_t)((H + j) * 32 + c.lane) * 2), "l"(b.x),
                         "l"(b.y)
                         : "memory");
        }
    }
    if (c.ghost_row) {
        const uint64_t* src = c.ghost_row + poff;
        ulonglong2 a[H], b[H];
        uint32_t it = 0;
        for (;;) {
            bool ok = true;
#pragma unroll
            for (int j = 0; j < H; ++j) {
                asm volatile("ld.volatile.global.v2.u64 {%0, %1}, [%2];\n"
                             : "=l"(a[j].x), "=l"(a[j].y)
                             : "l"(src + (size_t)(j * 32 + c.lane) * 2)
                             : "memory");
                asm volatile("ld.volatile.global.v2.u64 {%0, %1}, [%2];\n"
                             : "=l"(b[j].x), "=l"(b[j].y)
                             : "l"(src + (size_t)((H + j) * 32 + c.lane) * 2)
                             : "memory");
                ok = ok && (uint32_t)(a[j].x >> 32) == (uint32_t)m && (uint32_t)(a[j].y >> 32) == (uint32_t)m &&
                     (uint32_t)(b[j].x >> 32) == (uint32_t)m && (uint32_t)(b[j].y >> 32) == (uint32_t)m;
            }
            if (__all_sync(0xffffffffu, ok)) break;
            if (*c.failed || ++it == kMCSwapWaitLimit) {
                *c.failed = 1;
                break;
            }
        }
#pragma unroll
        for (int j = 0; j < H; ++j) {
            yu[j] = make_float2(__uint_as_float((uint32_t)a[j].x), __uint_as_float((uint32_t)a[j].y));
            yv[j] = make_float2(__uint_as_float((uint32_t)b[j].x), __uint_as_float((uint32_t)b[j].y));
        }
    }
}

// one step X -> Y of the warp's row (s: the step index of X; send: whether Y goes out)
template <int N, int C, int G, int WPC, int DRIFT>
__device__ __forceinline__ void mc_step(const MCCtx<N, C, G, WPC>& c, const GSCoef2& k, const float2 (&xu)[N / 64],
                                        const float2 (&xv)[N / 64], float2 (&yu)[N / 64], float2 (&yv)[N / 64],
                                        int s, bool send) {
    constexpr int H = N / 64;
    const int par = s & 1;
    rr_wait(c.bar(c.w, par), (uint32_t)(s >> 1) & 1u, c.failed);
    __syncwarp();
    if (c.lane == 0) rr_arm(c.bar(c.w, par), c.tx);   // the phase of step s + 2
    float2 au[H], av[H], bu[H], bv[H];
    rr_read_halo<H>(c.smem + (c.slot(c.w, par, 0, 0) - c.sbase), c.lane, au);
    rr_read_halo<H>(c.smem + (c.slot(c.w, par, 0, 1) - c.sbase), c.lane, av);
    rr_read_halo<H>(c.smem + (c.slot(c.w, par, 1, 0) - c.sbase), c.lane, bu);
    rr_read_halo<H>(c.smem + (c.slot(c.w, par, 1, 1) - c.sbase), c.lane, bv);
    rr_row<H, DRIFT>(k, au, xu, bu, av, xv, bv, yu, yv, c.lane);
    if (send) {
        if ((s + 1) % G == 0) mc_swap<N, C, G, WPC>(c, yu, yv, (s + 1) / G);
        const int np = par ^ 1;
        rr_send<H>(yu, yv, c.slot(c.up_w, np, 1, 0), c.slot(c.up_w, np, 1, 1), c.bar(c.up_w, np), c.up_remote,
                   c.up_rank, c.lane);
        rr_send<H>(yu, yv, c.slot(c.dn_w, np, 0, 0), c.slot(c.dn_w, np, 0, 1), c.bar(c.dn_w, np), c.dn_remote,
                   c.dn_rank, c.lane);
    }
}

// the ring neighbours, exchange roles and mbarriers of a warp's row (forward and
// adjoint alike); *row: the warp's lattice row, *band: whether it is a band row
template <int N, int C, int G, int WPC>
__device__ __forceinline__ void mc_setup(MCCtx<N, C, G, WPC>& c, unsigned char* smem_raw, uint64_t* xbuf,
                                         int* row, bool* band) {
    using S = MCShape<N, C, G, WPC>;
    constexpr int B = S::B;
    c.smem = smem_raw;
    c.sbase = smem_u32(smem_raw);
    c.lane = threadIdx.x & 31;
    c.w = threadIdx.x >> 5;
    const uint32_t rank = rr_ctarank();
    const int cl = (int)blockIdx.x / kRRCluster;
    c.up_remote = c.w == 0;
    c.dn_remote = c.w == WPC - 1;
    c.up_rank = c.up_remote ? (rank + kRRCluster - 1) % kRRCluster : rank;
    c.dn_rank = c.dn_remote ? (rank + 1) % kRRCluster : rank;
    c.up_w = c.up_remote ? WPC - 1 : c.w - 1;
    c.dn_w = c.dn_remote ? 0 : c.w + 1;
    c.failed = reinterpret_cast<volatile int*>(smem_raw + S::kHalo + WPC * 16);
    const int nremote = (int)c.up_remote + (int)c.dn_remote;
    c.tx = (uint32_t)nremote * 2u * S::kRow;
    // local row l of cluster cl is lattice row cl * B - G + l (periodic)
    const int l = (int)rank * WPC + c.w;
    *row = (cl * B - G + l + N) % N;
    *band = l >= G && l < G + B;
    // exchange roles: rows [G, 2G) feed the cluster above (side 0), rows [B, B + G) the
    // cluster below (side 1); ghost rows [0, G) come from the cluster above's side 1,
    // ghost rows [B + G, B + 2G) from the cluster below's side 0
    auto xrow = [&](int cluster, int side, int g) {
        return xbuf + (((size_t)cluster * 2 + side) * G + g) * S::kRowWords;
    };
    c.parity_stride = (size_t)C * 2 * G * S::kRowWords;
    c.src_row = nullptr;
    c.ghost_row = nullptr;
    if (l >= G && l < 2 * G) {
        c.src_row = xrow(cl, 0, l - G);
    } else if (l >= B && l < B + G) {
        c.src_row = xrow(cl, 1, l - B);
    } else if (l < G) {
        c.ghost_row = xrow((cl + C - 1) % C, 1, l);
    } else if (l >= B + G) {
        c.ghost_row = xrow((cl + 1) % C, 0, l - B - G);
    }
    if (c.lane == 0) {
        mbar_init(reinterpret_cast<uint64_t*>(smem_raw + (c.bar(c.w, 0) - c.sbase)), 1 + 32 * (2 - nremote));
        mbar_init(reinterpret_cast<uint64_t*>(smem_raw + (c.bar(c.w, 1) - c.sbase)), 1 + 32 * (2 - nremote));
        fence_mbar_init();
    }
    if (threadIdx.x == 0) *c.failed = 0;
}

template <int N, int C, int G, int WPC, int DRIFT>
__global__ void __launch_bounds__(32 * WPC, 1)
    k_gs_forward_mc(GSArgs<float> a, const float* __restrict__ u0, const float* __restrict__ v0,
                    float* __restrict__ uo, float* __restrict__ vo, float* __restrict__ trace, int trace_every,
                    uint64_t* __restrict__ xbuf) {
    using S = MCShape<N, C, G, WPC>;
    constexpr int H = S::H;
    constexpr int NN = N * N;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    MCCtx<N, C, G, WPC> c;
    int row;
    bool band;
    mc_setup<N, C, G, WPC>(c, smem_raw, xbuf, &row, &band);
    const int col0 = c.lane * 2 * H;
    const GSCoef2 k(a);
    float2 xu[H], xv[H], yu[H], yv[H];
    rr_load<H>(u0 + (size_t)row * N + col0, xu);
    rr_load<H>(v0 + (size_t)row * N + col0, xv);
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
        rr_send<H>(xu, xv, c.slot(c.up_w, 0, 1, 0), c.slot(c.up_w, 0, 1, 1), c.bar(c.up_w, 0), c.up_remote,
                   c.up_rank, c.lane);
        rr_send<H>(xu, xv, c.slot(c.dn_w, 0, 0, 0), c.slot(c.dn_w, 0, 0, 1), c.bar(c.dn_w, 0), c.dn_remote,
                   c.dn_rank, c.lane);
    }
    auto put_trace = [&](int s, const float2 (&pu)[H], const float2 (&pv)[H]) {
        if (trace != nullptr && band && s % every == 0) {
            float* du = trace + (size_t)(2 * (s / every)) * NN;
            rr_store<H>(du + (size_t)row * N + col0, pu);
            rr_store<H>(du + NN + (size_t)row * N + col0, pv);
        }
    };
    int s = 0;
    for (; s + 2 <= steps; s += 2) {      // two steps per iteration: X -> Y -> X without copies
        put_trace(s, xu, xv);
        mc_step<N, C, G, WPC, DRIFT>(c, k, xu, xv, yu, yv, s, true);
        put_trace(s + 1, yu, yv);
        mc_step<N, C, G, WPC, DRIFT>(c, k, yu, yv, xu, xv, s + 1, s + 2 < steps);
    }
    const bool odd = s < steps;
    if (odd) {
        put_trace(s, xu, xv);
        mc_step<N, C, G, WPC, DRIFT>(c, k, xu, xv, yu, yv, s, false);
    }
    __syncthreads();
    cluster_arrive();     // no CTA leaves while a neighbour may still address its shared memory
    cluster_wait();
    const bool bad = *c.failed != 0;
    if (bad && threadIdx.x == 0) atomicOr(&g_gs_fwd_err, 1);
    if (band) {
        const float nan = __int_as_float(0x7fc00000);
        float2 pu[H], pv[H];
#pragma unroll
        for (int j = 0; j < H; ++j) {
            pu[j] = bad ? make_float2(nan, nan) : (odd ? yu[j] : xu[j]);
            pv[j] = bad ? make_float2(nan, nan) : (odd ? yv[j] : xv[j]);
        }
        rr_store<H>(uo + (size_t)row * N + col0, pu);
        rr_store<H>(vo + (size_t)row * N + col0, pv);
    }
}

// ---- multi-cluster adjoint -------------------------------------------------------
// The transposed steps of a segment, last to first, over the same bands and ghost
// rows as the multi-cluster forward: the adjoint fields (lambda_u, lambda_v) of a
// warp's row stay in registers and are exchanged and swapped exactly like the forward
// rows (a ghost row's lambda goes stale from the ring's ends inwards just as a state
// row does).  The adjoint update needs the forward state only at the cell itself, so
// each warp reads its own row of the stored state from global memory, two steps
// ahead, into registers.  The parameter-gradient partial sums of ghost rows are
// dropped: every lattice cell is a band row of exactly one cluster.  The adjoint
// fields are bit-identical to the single-cluster adjoint's; the gradient sums differ
// from its only in the order of the float partial sums.

template <int N>
__device__ __forceinline__ void mc_adj_state(const float* __restrict__ states, int len, int q, int row, int col0,
                                             float2 (&su)[N / 64], float2 (&sv)[N / 64]) {
    constexpr int H = N / 64;
    constexpr size_t NN = (size_t)N * N;
    if (q >= len) return;
    const int j = len - 1 - q;   // adjoint step q uses stored state len - 1 - q
    rr_load<H>(states + (size_t)(2 * j) * NN + (size_t)row * N + col0, su);
    rr_load<H>(states + (size_t)(2 * j + 1) * NN + (size_t)row * N + col0, sv);
}

template <int N, int C, int G, int WPC, int DRIFT>
__device__ __forceinline__ void mc_adj_step(const MCCtx<N, C, G, WPC>& c, const GSCoef2& k,
                                            const float2 (&xa)[N / 64], const float2 (&xb)[N / 64],
                                            float2 (&ya)[N / 64], float2 (&yb)[N / 64], const float2 (&su)[N / 64],
                                            const float2 (&sv)[N / 64], int s, bool send, float2 t[6]) {
    constexpr int H = N / 64;
    const int par = s & 1;
    rr_wait(c.bar(c.w, par), (uint32_t)(s >> 1) & 1u, c.failed);
    __syncwarp();
    if (c.lane == 0) rr_arm(c.bar(c.w, par), c.tx);
    float2 ha[H], hb[H], la[H], lb[H];
    rr_read_halo<H>(c.smem + (c.slot(c.w, par, 0, 0) - c.sbase), c.lane, ha);
    rr_read_halo<H>(c.smem + (c.slot(c.w, par, 0, 1) - c.sbase), c.lane, hb);
    rr_read_halo<H>(c.smem + (c.slot(c.w, par, 1, 0) - c.sbase), c.lane, la);
    rr_read_halo<H>(c.smem + (c.slot(c.w, par, 1, 1) - c.sbase), c.lane, lb);
    rr_adj_row<H, DRIFT>(k, ha, xa, la, hb, xb, lb, su, sv, ya, yb, t, c.lane);
    if (send) {
        if ((s + 1) % G == 0) mc_swap<N, C, G, WPC>(c, ya, yb, (s + 1) / G);
        const int np = par ^ 1;
        rr_send<H>(ya, yb, c.slot(c.up_w, np, 1, 0), c.slot(c.up_w, np, 1, 1), c.bar(c.up_w, np), c.up_remote,
                   c.up_rank, c.lane);
        rr_send<H>(ya, yb, c.slot(c.dn_w, np, 0, 0), c.slot(c.dn_w, np, 0, 1), c.bar(c.dn_w, np), c.dn_remote,
                   c.dn_rank, c.lane);
    }
}

template <int N, int C, int G, int WPC, int DRIFT>
__global__ void __launch_bounds__(32 * WPC, 1)
    k_gs_adjoint_mc(GSArgs<float> a, const float* __restrict__ states, int len, const float* __restrict__ lu_in,
                    const float* __restrict__ lv_in, float* __restrict__ lu_out, float* __restrict__ lv_out,
                    double* __restrict__ grad, int* __restrict__ err, uint64_t* __restrict__ xbuf) {
    constexpr int H = N / 64;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double red[6][32];
    MCCtx<N, C, G, WPC> c;
    int row;
    bool band;
    mc_setup<N, C, G, WPC>(c, smem_raw, xbuf, &row, &band);
    const int col0 = c.lane * 2 * H;
    const GSCoef2 k(a);
    float2 xa[H], xb[H], ya[H], yb[H];
    rr_load<H>(lu_in + (size_t)row * N + col0, xa);
    rr_load<H>(lv_in + (size_t)row * N + col0, xb);
    // the forward state of the row for the even and the odd step of an iteration
    float2 eu[H], ev[H], ou[H], ov[H];
    mc_adj_state<N>(states, len, 0, row, col0, eu, ev);
    mc_adj_state<N>(states, len, 1, row, col0, ou, ov);
    __syncthreads();
    cluster_arrive();     // every CTA's mbarriers exist before anyone sends
    cluster_wait();
    if (len > 0) {
        if (c.lane == 0) {
            rr_arm(c.bar(c.w, 0), c.tx);
            rr_arm(c.bar(c.w, 1), c.tx);
        }
        rr_send<H>(xa, xb, c.slot(c.up_w, 0, 1, 0), c.slot(c.up_w, 0, 1, 1), c.bar(c.up_w, 0), c.up_remote,
                   c.up_rank, c.lane);
        rr_send<H>(xa, xb, c.slot(c.dn_w, 0, 0, 0), c.slot(c.dn_w, 0, 0, 1), c.bar(c.dn_w, 0), c.dn_remote,
                   c.dn_rank, c.lane);
    }
    // gradient partial sums: float over the two steps of an iteration, then double;
    // ghost rows' sums are dropped
    double g[6] = {0, 0, 0, 0, 0, 0};
    auto flush = [&](float2 (&t)[6]) {
#pragma unroll
        for (int q = 0; q < 6; ++q) {
            if (band) g[q] += (double)t[q].x + (double)t[q].y;
            t[q] = f2(0.f);
        }
    };
    float2 t[6] = {f2(0.f), f2(0.f), f2(0.f), f2(0.f), f2(0.f), f2(0.f)};
    int s = 0;
    for (; s + 2 <= len; s += 2) {
        mc_adj_step<N, C, G, WPC, DRIFT>(c, k, xa, xb, ya, yb, eu, ev, s, true, t);
        mc_adj_state<N>(states, len, s + 2, row, col0, eu, ev);
        mc_adj_step<N, C, G, WPC, DRIFT>(c, k, ya, yb, xa, xb, ou, ov, s + 1, s + 2 < len, t);
        mc_adj_state<N>(states, len, s + 3, row, col0, ou, ov);
        flush(t);
    }
    const bool odd = s < len;
    if (odd) {
        mc_adj_step<N, C, G, WPC, DRIFT>(c, k, xa, xb, ya, yb, eu, ev, s, false, t);
        flush(t);
    }
    g[4] = -g[4];      // gs_adj_update2s accumulates the drift sums negated
    g[5] = -g[5];
    __syncthreads();
    cluster_arrive();     // no CTA leaves while a neighbour may still address its shared memory
    cluster_wait();
    const bool bad = *c.failed != 0;
    if (bad && threadIdx.x == 0) atomicOr(err, 1);
    if (band) {
        const float nan = __int_as_float(0x7fc00000);
        float2 pa[H], pb[H];
#pragma unroll
        for (int j = 0; j < H; ++j) {
            pa[j] = bad ? make_float2(nan, nan) : (odd ? ya[j] : xa[j]);
            pb[j] = bad ? make_float2(nan, nan) : (odd ? yb[j] : xb[j]);
        }
        rr_store<H>(lu_out + (size_t)row * N + col0, pa);
        rr_store<H>(lv_out + (size_t)row * N + col0, pb);
    }
    grad_reduce(g, (double)a.dt, grad, red, (int)threadIdx.x, (int)blockDim.x);
}
