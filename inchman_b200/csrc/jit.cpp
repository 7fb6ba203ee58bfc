// Run-time compilation of model code with NVRTC (see jit.h).
#include "jit.h"

#include <dlfcn.h>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>
#include <cuda.h>
#include <nvrtc.h>
#include "host_common.h"
#include "individual.h"
#include "_jit_sources.h"

namespace gpgmp {

namespace {

// ---- NVRTC and driver entry points, resolved on first use ---------------------------
struct Api {
    bool tried = false, ok = false;
    std::string why;
    nvrtcResult (*createProgram)(nvrtcProgram*, const char*, const char*, int, const char* const*,
                                 const char* const*) = nullptr;
    nvrtcResult (*compileProgram)(nvrtcProgram, int, const char* const*) = nullptr;
    nvrtcResult (*getProgramLogSize)(nvrtcProgram, size_t*) = nullptr;
    nvrtcResult (*getProgramLog)(nvrtcProgram, char*) = nullptr;
    nvrtcResult (*getCUBINSize)(nvrtcProgram, size_t*) = nullptr;
    nvrtcResult (*getCUBIN)(nvrtcProgram, char*) = nullptr;
    nvrtcResult (*destroyProgram)(nvrtcProgram*) = nullptr;
    CUresult (*moduleLoadData)(CUmodule*, const void*) = nullptr;
    CUresult (*moduleGetFunction)(CUfunction*, CUmodule, const char*) = nullptr;
    CUresult (*launchKernel)(CUfunction, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned,
                             CUstream, void**, void**) = nullptr;
    CUresult (*funcSetAttribute)(CUfunction, CUfunction_attribute, int) = nullptr;
};

std::mutex g_mu;
Api g_api;
std::map<std::string, CUfunction> g_cache;

template <typename F>
bool sym(void* lib, const char* name, F* out) {
    *out = reinterpret_cast<F>(dlsym(lib, name));
    return *out != nullptr;
}

bool load_api(std::string* why) {
    if (g_api.tried) {
        *why = g_api.why;
        return g_api.ok;
    }
    g_api.tried = true;
    void* nv = dlopen("libnvrtc.so.12", RTLD_NOW | RTLD_LOCAL);
    if (!nv) nv = dlopen("libnvrtc.so", RTLD_NOW | RTLD_LOCAL);
    void* cu = dlopen("libcuda.so.1", RTLD_NOW | RTLD_LOCAL);
    if (!nv || !cu) {
        g_api.why = !nv ? "libnvrtc.so.12 not found" : "libcuda.so.1 not found";
        *why = g_api.why;
        return false;
    }
    bool ok = sym(nv, "nvrtcCreateProgram", &g_api.createProgram) &&
              sym(nv, "nvrtcCompileProgram", &g_api.compileProgram) &&
              sym(nv, "nvrtcGetProgramLogSize", &g_api.getProgramLogSize) &&
              sym(nv, "nvrtcGetProgramLog", &g_api.getProgramLog) &&
              sym(nv, "nvrtcGetCUBINSize", &g_api.getCUBINSize) && sym(nv, "nvrtcGetCUBIN", &g_api.getCUBIN) &&
              sym(nv, "nvrtcDestroyProgram", &g_api.destroyProgram) &&
              sym(cu, "cuModuleLoadData", &g_api.moduleLoadData) &&
              sym(cu, "cuModuleGetFunction", &g_api.moduleGetFunction) &&
              sym(cu, "cuLaunchKernel", &g_api.launchKernel) &&
              sym(cu, "cuFuncSetAttribute", &g_api.funcSetAttribute);
    if (!ok) g_api.why = "an NVRTC or driver entry point is missing";
    g_api.ok = ok;
    *why = g_api.why;
    return ok;
}

// fixed-width types and limits for the embedded headers under NVRTC
const char* kPrelude = R"GPGMPJIT(#pragma once
typedef unsigned int uint32_t;
typedef int int32_t;
typedef unsigned long long uint64_t;
typedef long long int64_t;
typedef unsigned char uint8_t;
#define INT_MAX 2147483647
#define INT32_MAX 2147483647
#define INFINITY __int_as_float(0x7f800000)
)GPGMPJIT";

int compile_module(const std::string& src, const std::vector<const char*>& names, std::vector<CUfunction>* outs);

// Compiles `src` for the current device (sm_100a) and returns kernel `name`.
int compile(const std::string& src, const char* name, CUfunction* out) {
    std::vector<CUfunction> fns;
    int rc = compile_module(src, {name}, &fns);
    if (rc == GPGMP_OK) *out = fns[0];
    return rc;
}

// Compiles `src` once and returns each of the kernels `names`.
int compile_module(const std::string& src, const std::vector<const char*>& names_in, std::vector<CUfunction>* outs) {
    std::string why;
    if (!load_api(&why)) return set_error(GPGMP_ERR_UNSUPPORTED, "run-time compilation unavailable: %s", why.c_str());
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaFree(nullptr) != cudaSuccess)
        return set_error(GPGMP_ERR_CUDA, "no CUDA context for run-time compilation");
    std::string key = std::to_string(dev) + '\0';
    for (const char* nm : names_in) key += std::string(nm) + '\0';
    key += src;
    outs->clear();
    bool cached = true;
    for (const char* nm : names_in) {
        auto it = g_cache.find(key + '\0' + nm);
        if (it == g_cache.end()) {
            cached = false;
            break;
        }
        outs->push_back(it->second);
    }
    if (cached) return GPGMP_OK;
    outs->clear();
    std::vector<const char*> names(kJitHeaderNames, kJitHeaderNames + kJitHeaderCount);
    std::vector<const char*> texts(kJitHeaderSources, kJitHeaderSources + kJitHeaderCount);
    names.push_back("gpgmp_rtc_prelude.h");
    texts.push_back(kPrelude);   // header names (the kernels' names are names_in)
    nvrtcProgram prog = nullptr;
    if (g_api.createProgram(&prog, src.c_str(), "gpgmp_model.cu", (int)names.size(), texts.data(), names.data()) !=
        NVRTC_SUCCESS)
        return set_error(GPGMP_ERR_INVALID, "nvrtcCreateProgram failed");
    const char* opts[] = {"-arch=sm_100a", "-fmad=false", "-std=c++17", "-default-device", "-DGPGMP_JIT"};
    const nvrtcResult rc = g_api.compileProgram(prog, 5, opts);
    if (rc != NVRTC_SUCCESS) {
        size_t n = 0;
        g_api.getProgramLogSize(prog, &n);
        std::string log(n, '\0');
        if (n) g_api.getProgramLog(prog, &log[0]);
        g_api.destroyProgram(&prog);
        if (log.size() > 1500) log.resize(1500);
        return set_error(GPGMP_ERR_INVALID, "model code does not compile: %s", log.c_str());
    }
    size_t n = 0;
    g_api.getCUBINSize(prog, &n);
    std::string cubin(n, '\0');
    g_api.getCUBIN(prog, &cubin[0]);
    g_api.destroyProgram(&prog);
    CUmodule mod = nullptr;
    CUresult cr = g_api.moduleLoadData(&mod, cubin.data());
    if (cr != CUDA_SUCCESS) return set_error(GPGMP_ERR_CUDA, "cuModuleLoadData: error %d", (int)cr);
    for (const char* nm : names_in) {
        CUfunction fn = nullptr;
        cr = g_api.moduleGetFunction(&fn, mod, nm);
        if (cr != CUDA_SUCCESS) return set_error(GPGMP_ERR_CUDA, "cuModuleGetFunction(%s): error %d", nm, (int)cr);
        g_cache[key + '\0' + nm] = fn;
        outs->push_back(fn);
    }
    return GPGMP_OK;
}

cudaError_t launch(CUfunction fn, unsigned grid, unsigned block, unsigned smem, cudaStream_t st, void** args) {
    if (smem > 48 * 1024 &&
        g_api.funcSetAttribute(fn, CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES, (int)smem) != CUDA_SUCCESS)
        return cudaErrorInvalidValue;
    const CUresult r = g_api.launchKernel(fn, grid, 1, 1, block, 1, 1, smem, (CUstream)st, args, nullptr);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorLaunchFailure;
}

constexpr int kJitSsaThreads = 128;

}  // namespace

int jit_ssa_kernel(const std::string& defines, const std::vector<std::string>& laws, JitFunction* out) {
    std::ostringstream s;
    s << "#include \"stoch_device.cuh\"\n"
      << defines << "\n"
      << "#define X(i) ((float)_x[(i) * _stride])\n"
      << "namespace gpgmp {\n"
      << "struct ModelHazard {\n"
      << "  __device__ __forceinline__ float operator()(const gpgmp_reaction* rt, int r, const int* _x, int _stride)"
      << " const {\n"
      << "    switch (r) {\n";
    for (size_t r = 0; r < laws.size(); ++r)
        if (!laws[r].empty()) s << "      case " << r << ": return (float)(" << laws[r] << ");\n";
    s << "      default: return hazard(rt[r], _x, _stride);\n"
      << "    }\n  }\n};\n}  // namespace gpgmp\n"
      << "struct JitPlanes { int* p[" << kMaxSpecies << "]; };\n"
      << "extern \"C\" __global__ void __launch_bounds__(" << kJitSsaThreads << ")\n"
      << "gpgmp_jit_ssa(JitPlanes planes, int S, int area, int R, const gpgmp_reaction* __restrict__ reactions,\n"
      << "              int nreac, unsigned seed, unsigned step_seed, float window, int* __restrict__ status,\n"
      << "              const unsigned* __restrict__ rmask, int rmask_words) {\n"
      << "  using namespace gpgmp;\n"
      << "  extern __shared__ __align__(16) unsigned char smem[];\n"
      << "  gpgmp_reaction* rt = reinterpret_cast<gpgmp_reaction*>(smem);\n"
      << "  int* xs = reinterpret_cast<int*>(smem + sizeof(gpgmp_reaction) * nreac);\n"
      << "  for (int i = threadIdx.x; i < nreac; i += blockDim.x) rt[i] = reactions[i];\n"
      << "  __syncthreads();\n"
      << "  const int64_t total = (int64_t)R * area;\n"
      << "  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;\n"
      << "  if (i >= total) return;\n"
      << "  const int r = (int)(i / area);\n"
      << "  const int c = (int)(i - (int64_t)r * area);\n"
      << "  int* x = xs + threadIdx.x;\n"
      << "  for (int s = 0; s < S; ++s) x[s * " << kJitSsaThreads << "] = planes.p[s][((int64_t)r * S + s) * area + c];\n"
      << "  Stream st;\n"
      << "  st.init(seed, (uint32_t)r, step_seed, (uint32_t)c, PH_SSA);\n"
      << "  int e;\n"
      << "  if (rmask) {\n"
      << "    CellReactions on;\n"
      << "    on.load(rmask, rmask_words, area, c);\n"
      << "    e = ssa_cell_h(rt, nreac, x, " << kJitSsaThreads
      << ", st, window, GatedHazard<ModelHazard>{ModelHazard{}, on});\n"
      << "  } else {\n"
      << "    e = ssa_cell_h(rt, nreac, x, " << kJitSsaThreads << ", st, window, ModelHazard{});\n"
      << "  }\n"
      << "  for (int s = 0; s < S; ++s) planes.p[s][((int64_t)r * S + s) * area + c] = x[s * " << kJitSsaThreads
      << "];\n"
      << "  if (e) atomicOr(&status[r], e);\n"
      << "}\n";
    std::lock_guard<std::mutex> lk(g_mu);
    CUfunction fn = nullptr;
    int rc = compile(s.str(), "gpgmp_jit_ssa", &fn);
    if (rc) return rc;
    *out = (JitFunction)fn;
    return GPGMP_OK;
}

cudaError_t launch_ssa_jit(JitFunction fn, const GridDesc& g, Planes planes, const gpgmp_reaction* d_reactions,
                           int nreac, uint32_t seed, uint32_t step_seed, float window, int32_t* d_status,
                           cudaStream_t st) {
    if (nreac <= 0) return cudaSuccess;
    int area = g.W * g.H, S = g.S, R = g.R;
    const int64_t total = (int64_t)R * area;
    const unsigned blocks = (unsigned)((total + kJitSsaThreads - 1) / kJitSsaThreads);
    const unsigned smem = (unsigned)(sizeof(gpgmp_reaction) * nreac + sizeof(int) * S * kJitSsaThreads);
    const uint32_t* rmask = g.rmask;
    int rmask_words = g.rmask_words;
    void* args[] = {&planes, &S,        &area,      &R,          (void*)&d_reactions, &nreac, &seed, &step_seed,
                    &window, &d_status, (void*)&rmask, &rmask_words};
    std::lock_guard<std::mutex> lk(g_mu);
    return launch((CUfunction)fn, blocks, kJitSsaThreads, smem, st, args);
}

int jit_drift_kernel(const std::string& defines, const std::string& code, JitFunction* out) {
    std::ostringstream s;
    s << "#include \"gpgmp_rtc_prelude.h\"\n"
      << "typedef float Real;\n"
      << "struct _species_t { int State; const int* SpeciesState; float MeanX;\n"
      << "                    float DiffusivityX; float DiffusivityY; float DriftX; float DriftY; };\n"
      << defines << "\n"
      << "struct JitStatePlanes { const int* p[" << kMaxSpecies << "]; };\n"
      // helpers.cl:38-87: neighbour differences of a species' counts, mirrored at the
      // edges (the reference bounds y by the grid width as well)
      << "__device__ __forceinline__ float _gp_cdx(const _species_t* sp, int x, int y, int W) {\n"
      << "  const int* d = sp->SpeciesState; if (!d) return 0.f;\n"
      << "  const int l = x > 0 ? d[(x - 1) + y * W] : d[(x + 1) + y * W];\n"
      << "  const int r = x < W - 1 ? d[(x + 1) + y * W] : d[(x - 1) + y * W];\n"
      << "  return (float)(r - l);\n}\n"
      << "__device__ __forceinline__ float _gp_cdy(const _species_t* sp, int x, int y, int W) {\n"
      << "  const int* d = sp->SpeciesState; if (!d) return 0.f;\n"
      << "  const int t = y > 0 ? d[x + (y - 1) * W] : d[x + (y + 1) * W];\n"
      << "  const int b = y < W - 1 ? d[x + (y + 1) * W] : d[x + (y - 1) * W];\n"
      << "  return (float)(b - t);\n}\n"
      << "extern \"C\" __global__ void gpgmp_jit_drift(int _W, int _H, int _S, int _species, float _L,\n"
      << "    float PhysicalSimTime, float* _dx, float* _dy, float* _rx, float* _ry, JitStatePlanes _planes,\n"
      << "    const float* _meanx, const float* _fields) {\n"
      << "  const int _area = _W * _H;\n"
      << "  const int GridModelWidth = _W, GridModelHeight = _H;\n"
      << "  const Real PhysicalModelWidth = _L, PhysicalModelHeight = _L;\n"
      << "  const Real PhysicalCellWidth = _L / (float)_W, PhysicalCellHeight = _L / (float)_H;\n"
      << "  for (int _c = blockIdx.x * blockDim.x + threadIdx.x; _c < _area; _c += gridDim.x * blockDim.x) {\n"
      << "    const int GridX = _c % _W, GridY = _c / _W;\n"
      << "    const Real PhysicalX = _L / (float)_W * ((float)GridX - (float)_W * 0.5f);\n"
      << "    const Real PhysicalY = _L / (float)_H * ((float)GridY - (float)_H * 0.5f);\n"
      << "    _species_t _sp[" << kMaxSpecies << "];\n"
      << "    for (int _s = 0; _s < _S; ++_s) {\n"
      << "      const long long _o = (long long)_s * _area + _c;\n"
      << "      const int* _pl = _planes.p[_s] ? _planes.p[_s] + (long long)_s * _area : nullptr;\n"
      << "      _sp[_s].State = _pl ? _pl[_c] : 0;\n"
      << "      _sp[_s].SpeciesState = _pl;\n"
      << "      _sp[_s].MeanX = _meanx ? _meanx[_s] : 0.f;\n"
      << "      _sp[_s].DiffusivityX = _dx[_o]; _sp[_s].DiffusivityY = _dy[_o];\n"
      << "      _sp[_s].DriftX = _rx[_o]; _sp[_s].DriftY = _ry[_o];\n"
      << "    }\n"
      << "#define SP(i) (&_sp[(i)])\n"
      << "#define F(f) (_fields[(long long)(f) * _area + _c])\n"
      << "#define getCentralDifferenceX(sp) _gp_cdx((sp), GridX, GridY, _W)\n"
      << "#define getCentralDifferenceY(sp) _gp_cdy((sp), GridX, GridY, _W)\n"
      << "#define getPhysicalX() (PhysicalX)\n#define getPhysicalY() (PhysicalY)\n"
      << "    _species_t* All = &_sp[_species];\n"
      << "    (void)GridX; (void)GridY; (void)PhysicalX; (void)PhysicalY; (void)PhysicalSimTime;\n"
      << "    (void)PhysicalModelWidth; (void)PhysicalModelHeight; (void)PhysicalCellWidth;\n"
      << "    (void)PhysicalCellHeight; (void)GridModelWidth; (void)GridModelHeight;\n"
      << "    {\n" << code << "\n    }\n"
      << "#undef SP\n#undef F\n#undef getCentralDifferenceX\n#undef getCentralDifferenceY\n"
      << "#undef getPhysicalX\n#undef getPhysicalY\n"
      << "    const long long _o = (long long)_species * _area + _c;\n"
      << "    _dx[_o] = All->DiffusivityX; _dy[_o] = All->DiffusivityY;\n"
      << "    _rx[_o] = All->DriftX; _ry[_o] = All->DriftY;\n"
      << "  }\n"
      << "}\n";
    std::lock_guard<std::mutex> lk(g_mu);
    CUfunction fn = nullptr;
    int rc = compile(s.str(), "gpgmp_jit_drift", &fn);
    if (rc) return rc;
    *out = (JitFunction)fn;
    return GPGMP_OK;
}

cudaError_t launch_drift_jit(JitFunction fn, const GridDesc& g, int species, float L, float sim_time, float* dx,
                             float* dy, float* rx, float* ry, const Planes* state, const float* meanx,
                             const float* fields, cudaStream_t st) {
    int W = g.W, H = g.H, S = g.S;
    const int area = W * H;
    const unsigned blocks = (unsigned)((area + 255) / 256 < 148 * 8 ? (area + 255) / 256 : 148 * 8);
    Planes planes{};
    if (state) planes = *state;
    void* args[] = {&W, &H, &S, &species, &L, &sim_time, &dx, &dy, &rx, &ry, &planes, (void*)&meanx, (void*)&fields};
    std::lock_guard<std::mutex> lk(g_mu);
    return launch((CUfunction)fn, blocks, 256, 0, st, args);
}

// The setField method (updateFields, Solver.cpp:583-653): per cell, X(i) is the count
// of species i as a float (written back truncated), F(f) field f of the cell.
int jit_field_kernel(const std::string& defines, const std::string& code, JitFunction* out) {
    std::ostringstream s;
    s << "#include \"gpgmp_rtc_prelude.h\"\n"
      << "typedef float Real;\n"
      << defines << "\n"
      << "struct JitMutPlanes { int* p[" << kMaxSpecies << "]; };\n"
      << "extern \"C\" __global__ void gpgmp_jit_fields(int _W, int _H, int _S, float _L, float deltat,\n"
      << "    float simtime, float* _fields, JitMutPlanes _planes) {\n"
      << "  const int _area = _W * _H;\n"
      << "  const int GridModelWidth = _W, GridModelHeight = _H;\n"
      << "  const Real PhysicalModelWidth = _L, PhysicalModelHeight = _L;\n"
      << "  const Real PhysicalCellWidth = _L / (float)_W, PhysicalCellHeight = _L / (float)_H;\n"
      << "  (void)GridModelWidth; (void)GridModelHeight; (void)PhysicalModelWidth; (void)PhysicalModelHeight;\n"
      << "  (void)PhysicalCellWidth; (void)PhysicalCellHeight; (void)deltat; (void)simtime;\n"
      << "  for (int _c = blockIdx.x * blockDim.x + threadIdx.x; _c < _area; _c += gridDim.x * blockDim.x) {\n"
      << "    const int GridX = _c % _W, GridY = _c / _W;\n"
      << "    (void)GridX; (void)GridY;\n"
      << "    float _x[" << kMaxSpecies << "];\n"
      << "    for (int _s = 0; _s < _S; ++_s) _x[_s] = (float)_planes.p[_s][(long long)_s * _area + _c];\n"
      << "#define X(i) (_x[(i)])\n"
      << "#define F(f) (_fields[(long long)(f) * _area + _c])\n"
      << "    {\n" << code << "\n    }\n"
      << "#undef X\n#undef F\n"
      << "    for (int _s = 0; _s < _S; ++_s) _planes.p[_s][(long long)_s * _area + _c] = (int)_x[_s];\n"
      << "  }\n"
      << "}\n";
    std::lock_guard<std::mutex> lk(g_mu);
    CUfunction fn = nullptr;
    int rc = compile(s.str(), "gpgmp_jit_fields", &fn);
    if (rc) return rc;
    *out = (JitFunction)fn;
    return GPGMP_OK;
}

cudaError_t launch_field_jit(JitFunction fn, const GridDesc& g, float L, float deltat, float simtime, float* fields,
                             const Planes& state, cudaStream_t st) {
    int W = g.W, H = g.H, S = g.S;
    const int area = W * H;
    const unsigned blocks = (unsigned)((area + 255) / 256 < 148 * 8 ? (area + 255) / 256 : 148 * 8);
    Planes planes = state;
    void* args[] = {&W, &H, &S, &L, &deltat, &simtime, &fields, &planes};
    std::lock_guard<std::mutex> lk(g_mu);
    return launch((CUfunction)fn, blocks, 256, 0, st, args);
}

// Individual species with model code (individual_device.cuh): the drift/diffusivity
// method and the new-individuals method inside the reference's environment -- the
// individual as All, every other species a zero dummy (IndividualSolver.cpp:210-238,
// 258-300), parameters and species names from `defines`, RANDOM a uniform draw.
int jit_ind_kernels(const std::string& defines, const std::string& drift_code, const std::string& newborn_code,
                    int num_species, IndKernels* out) {
    auto env = [&](std::ostringstream& s) {
        s << "    IndSpecies _d[" << (num_species > 0 ? num_species : 1) << "] = {};\n"
          << "    IndSpecies* All = &_me;\n"
          << "    const int GridX = _p.GridX, GridY = _p.GridY;\n"
          << "    const Real PhysicalX = _p.PhysicalX, PhysicalY = _p.PhysicalY, PhysicalSimTime = _p.PhysicalSimTime;\n"
          << "    const int GridModelWidth = _a.W, GridModelHeight = _a.H;\n"
          << "    const Real PhysicalModelWidth = _a.L, PhysicalModelHeight = _a.L;\n"
          << "    const Real PhysicalCellWidth = _a.L / (float)_a.W, PhysicalCellHeight = _a.L / (float)_a.H;\n"
          << "    (void)_d; (void)All; (void)GridX; (void)GridY; (void)PhysicalX; (void)PhysicalY;\n"
          << "    (void)PhysicalSimTime; (void)GridModelWidth; (void)GridModelHeight; (void)PhysicalModelWidth;\n"
          << "    (void)PhysicalModelHeight; (void)PhysicalCellWidth; (void)PhysicalCellHeight;\n"
          << "#define SP(i) ((i) == _a.species ? &_me : &_d[(i)])\n";
    };
    std::ostringstream s;
    s << "#include \"individual_device.cuh\"\n"
      << defines << "\n"
      << "typedef float Real;\n"
      << "typedef gpgmp::IndSpecies _species_t;\n"
      << "namespace gpgmp {\n"
      << "struct ModelIndDrift {\n"
      << "  __device__ __forceinline__ void operator()(IndSpecies& _me, const IndArgs& _a, const IndPos& _p) const {\n";
    env(s);
    s << "    {\n" << drift_code << "\n    }\n#undef SP\n  }\n};\n"
      << "struct ModelNewborn {\n"
      << "  __device__ __forceinline__ void operator()(IndSpecies& _me, const IndArgs& _a, const IndPos& _p,\n"
      << "                                             Stream& _st) const {\n";
    env(s);
    s << "#define RANDOM (::gpgmp::u01(_st.next()))\n"
      << "    {\n" << newborn_code << "\n    }\n#undef RANDOM\n#undef SP\n  }\n};\n"
      << "}  // namespace gpgmp\n"
      << "extern \"C\" __global__ void __launch_bounds__(256) gpgmp_ind_sweep(gpgmp::IndArgs a) {\n"
      << "  gpgmp::ind_sweep_body(a, gpgmp::ModelIndDrift());\n}\n"
      << "extern \"C\" __global__ void __launch_bounds__(256) gpgmp_ind_fields(gpgmp::IndArgs a) {\n"
      << "  gpgmp::ind_fields_body(a, gpgmp::ModelIndDrift());\n}\n"
      << "extern \"C\" __global__ void __launch_bounds__(256) gpgmp_ind_newborn(gpgmp::IndArgs a) {\n"
      << "  gpgmp::ind_newborn_body(a, gpgmp::ModelNewborn());\n}\n";
    std::lock_guard<std::mutex> lk(g_mu);
    std::vector<CUfunction> fns;
    int rc = compile_module(s.str(), {"gpgmp_ind_sweep", "gpgmp_ind_fields", "gpgmp_ind_newborn"}, &fns);
    if (rc) return rc;
    out->sweep = (JitFunction)fns[0];
    out->fields = (JitFunction)fns[1];
    out->newborn = (JitFunction)fns[2];
    out->newborn_active = !newborn_code.empty();
    return GPGMP_OK;
}

cudaError_t launch_ind_jit(JitFunction fn, const IndArgs& a, long long work, cudaStream_t st) {
    long long b = (work + 255) / 256;
    if (b < 1) b = 1;
    if (b > 148 * 8) b = 148 * 8;
    IndArgs copy = a;
    void* args[] = {&copy};
    std::lock_guard<std::mutex> lk(g_mu);
    return launch((CUfunction)fn, (unsigned)b, 256, 0, st, args);
}

}  // namespace gpgmp
