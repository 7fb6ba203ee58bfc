"""The device headers that the library compiles again at run time (NVRTC, csrc/jit.cpp)
compile with NVRTC and the library's options, checked on the CPU: NVRTC needs no GPU.
The kernels mirror what jit.cpp generates for a model with individual species (the
drift method and the new-individuals method), a drift method of count species and the
field method, each around the shared device bodies."""
import os
import re

import pytest

from inchman_b200 import build

nvrtc = pytest.importorskip("cuda.bindings.nvrtc")

OPTS = [b"-arch=sm_100a", b"-fmad=false", b"-std=c++17", b"-default-device", b"-DGPGMP_JIT"]


def _prelude():
    src = open(os.path.join(build.CSRC, "jit.cpp")).read()
    m = re.search(r'kPrelude = R"GPGMPJIT\((.*?)\)GPGMPJIT"', src, re.S)
    assert m, "prelude not found in jit.cpp"
    return m.group(1)


def _compile(src):
    names = [n.encode() for n, _ in build.JIT_HEADERS] + [b"gpgmp_rtc_prelude.h"]
    texts = [open(p, "rb").read() for _, p in build.JIT_HEADERS] + [_prelude().encode()]
    err, prog = nvrtc.nvrtcCreateProgram(src.encode(), b"gpgmp_model.cu", len(names), texts, names)
    assert err == nvrtc.nvrtcResult.NVRTC_SUCCESS
    (rc,) = nvrtc.nvrtcCompileProgram(prog, len(OPTS), OPTS)
    log = b""
    if rc != nvrtc.nvrtcResult.NVRTC_SUCCESS:
        _, n = nvrtc.nvrtcGetProgramLogSize(prog)
        log = b" " * n
        nvrtc.nvrtcGetProgramLog(prog, log)
    nvrtc.nvrtcDestroyProgram(prog)
    assert rc == nvrtc.nvrtcResult.NVRTC_SUCCESS, log.decode(errors="replace")


def test_individual_kernels_compile():
    _compile('''#include "individual_device.cuh"
typedef float Real;
namespace gpgmp {
struct ModelIndDrift {
  __device__ __forceinline__ void operator()(IndSpecies& _me, const IndArgs& _a, const IndPos& _p) const {
    _me.DiffusivityX = 0.5f + 0.01f * _me.State; _me.DriftX = -0.1f * _p.PhysicalX;
  }
};
struct ModelNewborn {
  __device__ __forceinline__ void operator()(IndSpecies& _me, const IndArgs& _a, const IndPos& _p,
                                             Stream& _st) const {
    _me.DiffusivityY = ::gpgmp::u01(_st.next());
  }
};
}  // namespace gpgmp
extern "C" __global__ void __launch_bounds__(256) gpgmp_ind_sweep(gpgmp::IndArgs a) {
  gpgmp::ind_sweep_body(a, gpgmp::ModelIndDrift());
}
extern "C" __global__ void __launch_bounds__(256) gpgmp_ind_fields(gpgmp::IndArgs a) {
  gpgmp::ind_fields_body(a, gpgmp::ModelIndDrift());
}
extern "C" __global__ void __launch_bounds__(256) gpgmp_ind_newborn(gpgmp::IndArgs a) {
  gpgmp::ind_newborn_body(a, gpgmp::ModelNewborn());
}
extern "C" __global__ void __launch_bounds__(256) gpgmp_ind_counts_timestep(gpgmp::IndArgs a, unsigned int* k) {
  gpgmp::ind_counts_timestep_body(a, 1.0f, gpgmp::kTsStochastic, 0.0f, k);
}
''')


def test_count_species_headers_compile():
    _compile('''#include "stoch_device.cuh"
extern "C" __global__ void probe(const float* D, const float* r, float* out, int n) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < n) out[c] = gpgmp::cell_timestep(D[c], r[c], 1.0f) + gpgmp::fpe_timestep(D[c], r[c], 1.0f, 0.5f)
                      + gpgmp::det_timestep(D[c], r[c], 1.0f);
}
''')
