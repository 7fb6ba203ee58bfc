// Run-time compilation of model code (NVRTC) into B200 kernels.
//
// The reference generates its OpenCL kernels from the model: custom propensity laws
// go into the Gillespie kernel (Solver.cpp:843-905) and the drift/diffusivity method
// becomes one kernel per species (Solver.cpp:643-777).  Here the same strings are
// compiled with NVRTC for sm_100a, together with the device headers the prebuilt
// kernels use (embedded at build time), so a custom-law SSA runs exactly the prebuilt
// SSA's code with only the hazard replaced.  NVRTC and the driver API are opened with
// dlopen on first use; a library user without custom code never needs them.
#pragma once
#include <string>
#include <vector>
#include <cuda_runtime.h>
#include "kernels.h"

namespace gpgmp {

// Opaque compiled kernel (a CUfunction of a module kept for the life of the process).
typedef void* JitFunction;

// SSA reaction-window kernel whose reaction r has the propensity custom_laws[r] (a C
// expression in X(i) = count of species i as float and the caller's defines), or the
// mass-action hazard where custom_laws[r] is empty.  Cached per device and source.
int jit_ssa_kernel(const std::string& defines, const std::vector<std::string>& custom_laws, JitFunction* out);
cudaError_t launch_ssa_jit(JitFunction fn, const GridDesc& g, Planes planes, const gpgmp_reaction* d_reactions,
                           int nreac, uint32_t seed, uint32_t step_seed, float window, int32_t* d_status,
                           cudaStream_t st);

// Drift/diffusivity kernel of the user method `code` (statements on All / SP(i)).
int jit_drift_kernel(const std::string& defines, const std::string& code, JitFunction* out);
// Evaluates the method for `species` over the grid: reads and writes the field
// arrays [S][H][W].  state: the current plane base of each species (realisation 0's
// counts are read), NULL for none; meanx: MeanX of each species (moments), NULL for 0;
// fields: the field parameters [F][H][W] (F(f) in the code), NULL for none.
cudaError_t launch_drift_jit(JitFunction fn, const GridDesc& g, int species, float L, float sim_time, float* dx,
                             float* dy, float* rx, float* ry, const Planes* state, const float* meanx,
                             const float* fields, cudaStream_t st);
// The setField method (see jit.cpp): one pass over the grid of realisation 0.
int jit_field_kernel(const std::string& defines, const std::string& code, JitFunction* out);
cudaError_t launch_field_jit(JitFunction fn, const GridDesc& g, float L, float deltat, float simtime, float* fields,
                             const Planes& state, cudaStream_t st);

}  // namespace gpgmp
