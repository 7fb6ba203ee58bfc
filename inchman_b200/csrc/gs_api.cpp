// C ABI of the Gray-Scott forward and adjoint solvers (gray_scott.cu).
//
// The adjoint uses two-level checkpointing: the forward pass keeps the state every
// checkpoint_every steps; the backward pass walks the segments last to first,
// recomputes each segment's states from its checkpoint into a work buffer (one
// forward launch, on a side stream, up to two segments ahead), then runs the
// transposed steps over them (one adjoint launch on the caller's stream).  Memory:
// ceil(steps/c) + 2c states; time: the forward solve plus the adjoint steps, with
// the recomputation overlapped.
#include <algorithm>
#include <cstring>
#include <mutex>
#include <vector>
#include <cuda_runtime.h>
#include "gs_kernels.h"
#include "host_common.h"
#include "../../include/gpgmp_c.h"

using namespace gpgmp;

namespace {

#define CK(expr)                                                                                              \
    do {                                                                                                      \
        cudaError_t e_ = (expr);                                                                              \
        if (e_ != cudaSuccess) return set_error(GPGMP_ERR_CUDA, "%s: %s", #expr, cudaGetErrorString(e_));    \
    } while (0)

int check(const gpgmp_gs_params* p, int elem_bytes) {
    if (!p) return set_error(GPGMP_ERR_INVALID, "params is NULL");
    if (p->n <= 2 || p->steps < 0) return set_error(GPGMP_ERR_INVALID, "n %d steps %d", p->n, p->steps);
    int cl = p->cluster > 0 ? p->cluster : gs_cluster_size(p->n, elem_bytes);
    if (cl <= 0 || cl > 16 || p->n % cl)
        return set_error(GPGMP_ERR_UNSUPPORTED, "lattice %d does not fit one thread-block cluster", p->n);
    if ((size_t)elem_bytes * 4 * (size_t)(p->n / cl + 2) * p->n > 227 * 1024)
        return set_error(GPGMP_ERR_UNSUPPORTED, "lattice %d needs more shared memory per CTA than a B200 has", p->n);
    return GPGMP_OK;
}

GSParams to_params(const gpgmp_gs_params* p) {
    GSParams g;
    g.n = p->n; g.steps = p->steps;
    g.F = p->F; g.k = p->k; g.Du = p->Du; g.Dv = p->Dv; g.vx = p->vx; g.vy = p->vy; g.dt = p->dt;
    g.cluster = p->cluster;
    g.variant = p->variant;
    return g;
}

// the automatic interval: 100 steps in float32 (shorter segments add launches to a
// latency-bound adjoint: 3.05 / 3.30 / 3.79 x the forward at 100 / 50 / 25 steps);
// 25 in float64, whose two 25-state segment buffers (50 MB at 256^2) stay in L2 while
// the adjoint reads them back (3.11 / 3.28 / 3.70 at 25 / 50 / 100 steps, the 50-step
// buffers at the edge of L2 and 3.78 in some runs)
int ck_every(const gpgmp_gs_params* p, int elem_bytes) {
    return p->checkpoint_every > 0 ? p->checkpoint_every : (elem_bytes == 8 ? 25 : 100);
}

template <typename T>
int forward(const gpgmp_gs_params* p, const T* u0, const T* v0, T* u, T* v, T* ckpt, void* stream) {
    int rc = check(p, sizeof(T));
    if (rc) return rc;
    GSParams g = to_params(p);
    CK(gs_forward<T>(g, u0, v0, u, v, ckpt, ck_every(p, (int)sizeof(T)), (cudaStream_t)stream));
    return GPGMP_OK;
}

// Side stream and events of the backward pipeline, one set per device, created on
// first use and kept for the life of the process.  The mutex also makes the
// enqueue of one backward pass atomic with respect to another host thread's.
struct GSPipe {
    cudaStream_t side = nullptr;
    cudaEvent_t start = nullptr, rec[2] = {nullptr, nullptr}, adj[2] = {nullptr, nullptr};
};
std::mutex& pipe_mutex() {
    static std::mutex m;
    return m;
}
int side_pipe(GSPipe** out) {
    static GSPipe pipes[64];
    int dev = 0;
    CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return set_error(GPGMP_ERR_UNSUPPORTED, "device ordinal %d", dev);
    GSPipe& q = pipes[dev];
    if (!q.side) {
        CK(cudaStreamCreateWithFlags(&q.side, cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&q.start, cudaEventDisableTiming));
        for (int b = 0; b < 2; ++b) {
            CK(cudaEventCreateWithFlags(&q.rec[b], cudaEventDisableTiming));
            CK(cudaEventCreateWithFlags(&q.adj[b], cudaEventDisableTiming));
        }
    }
    *out = &q;
    return GPGMP_OK;
}

// Backward pass.  The recomputation of a segment's states depends only on its
// checkpoint, so it runs on a side stream up to two segments ahead of the adjoint
// steps on the caller's stream (two segment buffers; a buffer is refilled after
// the adjoint launch that read it).  The two run concurrently on different SMs.
template <typename T>
int adjoint(const gpgmp_gs_params* p, const T* ckpt, const T* lu, const T* lv, T* gu, T* gv, double* grad6,
            void* work, void* stream) {
    int rc = check(p, sizeof(T));
    if (rc) return rc;
    if (!ckpt || !lu || !lv || !gu || !gv || !grad6 || !work) return set_error(GPGMP_ERR_INVALID, "NULL argument");
    cudaStream_t st = (cudaStream_t)stream;
    const int c = ck_every(p, (int)sizeof(T));
    const size_t nn = (size_t)p->n * p->n;
    T* segb[2] = {(T*)work, (T*)work + (size_t)2 * c * nn};   // c states, 2 nn each
    T* fin[2] = {segb[1] + (size_t)2 * c * nn, segb[1] + (size_t)2 * c * nn + 2 * nn};   // recomputed end states
    T* lam = fin[1] + 2 * nn;                // two adjoint buffers (u, v) x 2
    T* la[2] = {lam, lam + 2 * nn};
    int* err = (int*)(lam + 4 * nn);         // status word: a bounded in-kernel wait gave up
    CK(cudaMemsetAsync(grad6, 0, 6 * sizeof(double), st));
    CK(cudaMemsetAsync(err, 0, sizeof(int), st));
    CK(cudaMemcpyAsync(la[0], lu, nn * sizeof(T), cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(la[0] + nn, lv, nn * sizeof(T), cudaMemcpyDeviceToDevice, st));
    const int nseg = (p->steps + c - 1) / c;
    if (nseg == 0) {
        CK(cudaMemcpyAsync(gu, lu, nn * sizeof(T), cudaMemcpyDeviceToDevice, st));
        CK(cudaMemcpyAsync(gv, lv, nn * sizeof(T), cudaMemcpyDeviceToDevice, st));
        return GPGMP_OK;
    }
    GSParams g = to_params(p);
    // float32 under the automatic choice, where the forward is the multi-cluster kernel:
    // the segments are recomputed on two clusters (32 SMs, variant 40) and the adjoint
    // runs on four (64 SMs), so both fit on the chip at once (backward 10.6 ms, against
    // 12.0 ms with the single-cluster recomputation, 15.2 ms with the multi-cluster
    // recomputation and the single-cluster adjoint, 256^2, 10,000 steps); every pairing
    // gives the same bits of lambda.  Where four clusters are resident at once two are;
    // the adjoint never waits on the recomputation beside it, so a recomputation that
    // finds only part of the chip free waits (bounded) for the adjoint's SMs, no longer
    GSParams gr = g, ga = g;
    if (sizeof(T) == 4 && g.variant == 0) {
        int v = 0;
        CK(gs_auto_variant(p->n, p->vx != 0.0 || p->vy != 0.0, &v));
        if (v >= 40) {
            gr.variant = 40;
            ga.variant = v;
        }
    }
    std::lock_guard<std::mutex> lk(pipe_mutex());
    GSPipe* pp = nullptr;
    rc = side_pipe(&pp);
    if (rc) return rc;
    CK(cudaEventRecord(pp->start, st));               // checkpoints and inputs are ready
    CK(cudaStreamWaitEvent(pp->side, pp->start, 0));
    bool used[2] = {false, false};
    auto seg_len = [&](int sgi) { return std::min(c, p->steps - sgi * c); };
    auto recompute = [&](int sgi) -> int {
        const int b = sgi & 1;
        if (used[b]) CK(cudaStreamWaitEvent(pp->side, pp->adj[b], 0));
        GSParams gf = gr;
        gf.steps = seg_len(sgi);
        const T* cku = ckpt + (size_t)2 * sgi * nn;
        // states before steps 0..len-1 of the segment into segb[b]
        CK(gs_forward<T>(gf, cku, cku + nn, fin[b], fin[b] + nn, segb[b], 1, pp->side));
        CK(cudaEventRecord(pp->rec[b], pp->side));
        return GPGMP_OK;
    };
    int next = nseg - 1;
    for (int q = 0; q < 2 && next >= 0; ++q, --next) {
        rc = recompute(next);
        if (rc) return rc;
    }
    int cur = 0;
    for (int sgi = nseg - 1; sgi >= 0; --sgi) {
        const int b = sgi & 1;
        CK(cudaStreamWaitEvent(st, pp->rec[b], 0));
        T* ou = sgi == 0 ? gu : la[1 - cur];
        T* ov = sgi == 0 ? gv : la[1 - cur] + nn;
        CK(gs_adjoint_segment<T>(ga, segb[b], seg_len(sgi), la[cur], la[cur] + nn, ou, ov, grad6, err, st));
        CK(cudaEventRecord(pp->adj[b], st));
        used[b] = true;
        cur = 1 - cur;
        if (next >= 0) {
            rc = recompute(next--);
            if (rc) return rc;
        }
    }
    return GPGMP_OK;
}

}  // namespace

extern "C" {

int gpgmp_gs_buffer_sizes(const gpgmp_gs_params* p, int32_t elem_bytes, size_t* ck_bytes, size_t* work_bytes) {
    if (!p || !ck_bytes || !work_bytes) return set_error(GPGMP_ERR_INVALID, "NULL argument");
    if (elem_bytes != 4 && elem_bytes != 8) return set_error(GPGMP_ERR_INVALID, "elem_bytes %d", elem_bytes);
    const int c = ck_every(p, elem_bytes);
    const size_t nn = (size_t)p->n * p->n;
    const size_t nseg = (size_t)((p->steps + c - 1) / c);
    *ck_bytes = std::max<size_t>(1, nseg) * 2 * nn * elem_bytes;
    // two segment buffers, two recomputed end states, two adjoint buffers, status word
    *work_bytes = ((size_t)4 * c * nn + 8 * nn) * elem_bytes + 16;
    return GPGMP_OK;
}

int gpgmp_gs_forward_f32(const gpgmp_gs_params* p, const float* u0, const float* v0, float* u, float* v, float* ck,
                         void* stream) {
    return forward<float>(p, u0, v0, u, v, ck, stream);
}
int gpgmp_gs_forward_f64(const gpgmp_gs_params* p, const double* u0, const double* v0, double* u, double* v,
                         double* ck, void* stream) {
    return forward<double>(p, u0, v0, u, v, ck, stream);
}
int gpgmp_gs_adjoint_f32(const gpgmp_gs_params* p, const float* ck, const float* lu, const float* lv, float* gu,
                         float* gv, double* grad6, void* work, void* stream) {
    return adjoint<float>(p, ck, lu, lv, gu, gv, grad6, work, stream);
}
int gpgmp_gs_adjoint_f64(const gpgmp_gs_params* p, const double* ck, const double* lu, const double* lv, double* gu,
                         double* gv, double* grad6, void* work, void* stream) {
    return adjoint<double>(p, ck, lu, lv, gu, gv, grad6, work, stream);
}

int gpgmp_gs_forward_batch_f32(const gpgmp_gs_params* p, int32_t batch, const double* member_params,
                               const float* u0, const float* v0, float* u, float* v, void* stream) {
    int rc = check(p, 4);
    if (rc) return rc;
    if (batch <= 0 || !u0 || !v0 || !u || !v) return set_error(GPGMP_ERR_INVALID, "bad argument");
    if ((p->cluster != 0 && p->cluster != 16) || (p->variant != 0 && p->variant != 3 && p->variant <= 10))
        return set_error(GPGMP_ERR_UNSUPPORTED, "batched solves use the register-resident kernel");
    std::vector<GSBatchMember> m(batch);
    for (int b = 0; b < batch; ++b) {
        const double* q = member_params ? member_params + 6 * (size_t)b : nullptr;
        m[b] = GSBatchMember{q ? q[0] : p->F, q ? q[1] : p->k, q ? q[2] : p->Du, q ? q[3] : p->Dv,
                             q ? q[4] : p->vx, q ? q[5] : p->vy};
    }
    cudaError_t e = gs_forward_batch_f32(to_params(p), batch, m.data(), u0, v0, u, v, (cudaStream_t)stream);
    if (e == cudaErrorInvalidValue)
        return set_error(GPGMP_ERR_UNSUPPORTED, "lattice %d has no register-resident kernel", p->n);
    CK(e);
    return GPGMP_OK;
}

int gpgmp_gs_batch_capacity(int32_t n, int32_t* lattices) {
    if (!lattices) return set_error(GPGMP_ERR_INVALID, "NULL argument");
    int c = 0;
    cudaError_t e = gs_batch_capacity(n, &c);
    if (e == cudaErrorInvalidValue) return set_error(GPGMP_ERR_UNSUPPORTED, "lattice %d", n);
    CK(e);
    *lattices = c;
    return GPGMP_OK;
}

int gpgmp_gs_auto_variant(int32_t n, int32_t drift, int32_t* variant) {
    if (!variant) return set_error(GPGMP_ERR_INVALID, "NULL argument");
    if (n <= 2) return set_error(GPGMP_ERR_INVALID, "n %d", n);
    int v = 0;
    CK(gs_auto_variant(n, drift != 0, &v));
    *variant = v;
    return GPGMP_OK;
}

int gpgmp_gs_status(int32_t* flags) {
    if (!flags) return set_error(GPGMP_ERR_INVALID, "NULL argument");
    CK(cudaDeviceSynchronize());
    int v = 0;
    CK(gs_forward_status(&v, true));
    *flags = v;
    return GPGMP_OK;
}

}  // extern "C"

namespace {
// Device buffers of one host-buffer call, returned to the pool in stream order on
// every exit path.
template <int N>
struct PoolBuffers {
    explicit PoolBuffers(cudaStream_t s) : st(s) {}
    ~PoolBuffers() {
        for (void* q : p) gpgmp::pool_free(q, st);
    }
    cudaStream_t st;
    void* p[N] = {};
};
}  // namespace

extern "C" {

int gpgmp_gs_forward_host(const gpgmp_gs_params* p, const float* u0, const float* v0, float* u, float* v) {
    int rc = check(p, 4);
    if (rc) return rc;
    if (!u0 || !v0 || !u || !v) return set_error(GPGMP_ERR_INVALID, "NULL argument");
    const size_t nn = (size_t)p->n * p->n, bytes = nn * sizeof(float);
    cudaStream_t st = nullptr;
    PoolBuffers<1> buf(st);
    float* d = nullptr;
    CK(pool_alloc((void**)&d, 4 * bytes, st));
    buf.p[0] = d;
    CK(cudaMemcpyAsync(d, u0, bytes, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(d + nn, v0, bytes, cudaMemcpyHostToDevice, st));
    rc = forward<float>(p, d, d + nn, d + 2 * nn, d + 3 * nn, nullptr, st);
    if (rc == GPGMP_OK) {
        CK(cudaMemcpyAsync(u, d + 2 * nn, bytes, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(v, d + 3 * nn, bytes, cudaMemcpyDeviceToHost, st));
    }
    CK(cudaStreamSynchronize(st));
    if (rc == GPGMP_OK) {
        int bad = 0;
        CK(gs_forward_status(&bad, true));
        if (bad) return set_error(GPGMP_ERR_TIMEOUT, "a bounded halo wait in the forward solve gave up");
    }
    return rc;
}

int gpgmp_gs_loss_grad_host(const gpgmp_gs_params* p, const float* u0, const float* v0, const float* ut,
                            const float* vt, double* loss, double* grad6) {
    int rc = check(p, 4);
    if (rc) return rc;
    if (!u0 || !v0 || !ut || !vt || !loss || !grad6) return set_error(GPGMP_ERR_INVALID, "NULL argument");
    const size_t nn = (size_t)p->n * p->n, bytes = nn * sizeof(float);
    size_t ckb = 0, wb = 0;
    gpgmp_gs_buffer_sizes(p, 4, &ckb, &wb);
    cudaStream_t st = nullptr;
    PoolBuffers<4> buf(st);
    float *d = nullptr, *ck = nullptr, *work = nullptr;
    double* dg = nullptr;
    CK(pool_alloc((void**)&d, 8 * bytes, st));
    buf.p[0] = d;
    CK(pool_alloc((void**)&ck, ckb, st));
    buf.p[1] = ck;
    CK(pool_alloc((void**)&work, wb, st));
    buf.p[2] = work;
    CK(pool_alloc((void**)&dg, 6 * sizeof(double), st));
    buf.p[3] = dg;
    CK(cudaMemcpyAsync(d, u0, bytes, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(d + nn, v0, bytes, cudaMemcpyHostToDevice, st));
    rc = forward<float>(p, d, d + nn, d + 2 * nn, d + 3 * nn, ck, st);
    if (rc) return rc;
    std::vector<float> un(nn), vn(nn);
    CK(cudaMemcpyAsync(un.data(), d + 2 * nn, bytes, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(vn.data(), d + 3 * nn, bytes, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    double L = 0;
    std::vector<float> lu(nn), lv(nn);
    for (size_t i = 0; i < nn; ++i) {
        const double a = (double)un[i] - ut[i], b = (double)vn[i] - vt[i];
        L += a * a + b * b;
        lu[i] = (float)(2.0 * a);
        lv[i] = (float)(2.0 * b);
    }
    CK(cudaMemcpyAsync(d + 4 * nn, lu.data(), bytes, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(d + 5 * nn, lv.data(), bytes, cudaMemcpyHostToDevice, st));
    rc = adjoint<float>(p, ck, d + 4 * nn, d + 5 * nn, d + 6 * nn, d + 7 * nn, dg, work, st);
    if (rc) return rc;
    int err = 0;
    CK(cudaMemcpyAsync(grad6, dg, 6 * sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(&err, (char*)work + wb - 16, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (err) return set_error(GPGMP_ERR_TIMEOUT, "a bounded wait for a TMA copy in the adjoint gave up");
    CK(gs_forward_status(&err, true));
    if (err) return set_error(GPGMP_ERR_TIMEOUT, "a bounded halo wait in the forward solve gave up");
    *loss = L;
    return GPGMP_OK;
}

}  // extern "C"
