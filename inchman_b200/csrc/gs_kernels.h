// Launchers of the Gray-Scott cluster kernels (gray_scott.cu).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace gpgmp {

struct GSParams {
    int n, steps;
    double F, k, Du, Dv, vx, vy, dt;
    int cluster;   // CTAs per cluster, 0 = 16 where the lattice fits, else the smallest that fits
    int variant;   // 0 automatic, 1 one cell per iteration, 2 shared-memory column walk,
                   // 3 register-resident (float32), 10 + w register-resident with w warps per CTA
};

// per-lattice parameters of a batched forward solve
struct GSBatchMember {
    double F, k, Du, Dv, vx, vy;
};
// batch independent float32 n x n lattices (u0/v0/u/v: [batch][n][n]) with their own
// parameters (p.n, p.steps, p.dt shared), one 16-CTA cluster each, in one launch of
// the register-resident kernel
cudaError_t gs_forward_batch_f32(const GSParams& p, int batch, const GSBatchMember* members, const float* u0,
                                 const float* v0, float* u, float* v, cudaStream_t st);

// how many lattices of side n a batched launch runs at the same time on this device
// (16-CTA clusters that fit at once)
cudaError_t gs_batch_capacity(int n, int* clusters);
// the float32 family variant 0 resolves to for an n x n lattice on the current device
cudaError_t gs_auto_variant(int n, bool drift, int* variant);

// reads (and with clear, resets) the device word that the register-resident forward
// kernel sets when one of its bounded waits gave up; synchronous
cudaError_t gs_forward_status(int* out, bool clear);

// cluster size (<= 16) for an n x n lattice of elem_bytes values: 16 when the
// lattice splits evenly into 16 slabs that fit, else the smallest that fits
int gs_cluster_size(int n, int elem_bytes);

// p.steps explicit steps from (u0, v0) into (u, v).  If trace is not NULL it receives
// the state before every step s with s % trace_every == 0:
// trace[2 (s / trace_every) n^2 ...] = u_s, the next n^2 values v_s.
template <typename T>
cudaError_t gs_forward(const GSParams& p, const T* u0, const T* v0, T* u, T* v, T* trace, int trace_every,
                       cudaStream_t st);

// Adjoint of `len` steps whose input states are states[j] (j = 0..len-1, layout as
// trace above): lam_out = J^T ... J^T lam_in; adds dt-weighted parameter gradients
// (F, k, Du, Dv, vx, vy) into grad[0..5].
// err: device word set non-zero if a bounded wait inside the kernel gave up.
template <typename T>
cudaError_t gs_adjoint_segment(const GSParams& p, const T* states, int len, const T* lu_in, const T* lv_in, T* lu_out,
                               T* lv_out, double* grad, int* err, cudaStream_t st);

}  // namespace gpgmp
