// Host-side launchers of the CUDA kernels (implemented in the .cu files).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "../../include/gpgmp_c.h"

namespace gpgmp {

constexpr int kMaxSpecies = 32;
constexpr int kNumDiffusionTiles = 6;     // diffusion tile shapes (diffusion_tile_shape)
constexpr int kNumSsaThreadChoices = 3;   // SSA block sizes (ssa_thread_choice)

// Per-species plane bases: species s of realisation r, cell c lives at
// planes.p[s][(r * S + s) * area + c].  The two state buffers alternate per
// species because the fused diffusion kernels write out of place.
struct Planes {
    int32_t* p[kMaxSpecies];
};
struct FPlanes {
    float* p[kMaxSpecies];
};

struct GridDesc {
    int W, H, S, R;          // grid, species, realisations
    int bmask[4];
    // localised reactions: [rmask_words][W * H] bits, bit r % 32 of word r / 32 of a
    // cell set where reaction r may fire; NULL when every reaction fires everywhere
    const uint32_t* rmask;
    int rmask_words;
    // launch shapes: index of the diffusion tile shape and of the SSA block size (0:
    // the defaults, 32 x 16 cells and 128 threads); the results do not depend on them
    int tile;
    int ssa_threads;
};
// the tile of shape index i is w x h cells; SSA block size choice i is that many threads
void diffusion_tile_shape(int index, int* w, int* h);
int ssa_thread_choice(int index);

cudaError_t launch_init_poisson(const GridDesc& g, Planes planes, uint32_t seed, const float* d_lambda,
                                cudaStream_t st);
cudaError_t launch_ssa(const GridDesc& g, Planes planes, const gpgmp_reaction* d_reactions, int nreac,
                       uint32_t seed, uint32_t step_seed, float window, int32_t* d_status, cudaStream_t st);
cudaError_t launch_homog_diffuse(const GridDesc& g, const int32_t* in, int32_t* out, int species, uint32_t seed,
                                 uint32_t step_seed, float pmove, cudaStream_t st);
cudaError_t launch_source(const GridDesc& g, int32_t* plane_base, int species, uint32_t seed, uint32_t step_seed,
                          int boundary, int count, float pi, cudaStream_t st);
// fpe: the FPE discretisation's jump probabilities (stochastic_inhomogeneous_fpe)
cudaError_t launch_sweep(const GridDesc& g, const int32_t* in, int32_t* out, int species, int sweep_y,
                         uint32_t seed, uint32_t step_seed, const float* d_D, const float* d_r, float dt, float dx,
                         cudaStream_t st, int fpe = 0);
// kind: 0 stochastic drift-diffusion, 1 FPE (uses stay), 2 deterministic
// MeanX of one species plane (the reference's moments): *d_meanx on the device
cudaError_t launch_moments(const int32_t* plane, int W, int H, float L, unsigned long long* d_sums, float* d_meanx,
                           cudaStream_t st);
cudaError_t launch_timestep(int area, const float* d_D, const float* d_r, float dx, uint32_t* d_min_key,
                            cudaStream_t st, int kind = 0, float stay = 0.f);
cudaError_t launch_diffusivity_drift(const GridDesc& g, int species, int method, const float* params, float L,
                                     float* dx, float* dy, float* rx, float* ry, cudaStream_t st);

// deterministic reference-compatible path (float state)
cudaError_t launch_det_diffuse(const GridDesc& g, const float* in, float* out, const float* d_D, float dt,
                               float dx2, cudaStream_t st);
cudaError_t launch_rk4(const GridDesc& g, float* state, const gpgmp_reaction* d_reactions, int nreac,
                       float deltat, cudaStream_t st);
// inhomogeneous deterministic drift-diffusion, one species, one direction (out of place;
// `out` receives the whole state)
cudaError_t launch_det_sweep(const GridDesc& g, const float* in, float* out, int species, int sweep_y,
                             const float* d_D, const float* d_r, float dt, float dx, cudaStream_t st);
// alpha-QSS reaction window (literal: the reference's corrector coefficient as printed)
cudaError_t launch_aqss(const GridDesc& g, float* state, const gpgmp_reaction* d_reactions, int nreac, float deltat,
                        int literal, int32_t* d_status, cudaStream_t st);

// order-preserving float <-> uint key for atomicMin over floats
inline float key_to_float(uint32_t k) {
    uint32_t b = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
    float f;
    static_assert(sizeof(f) == 4, "float");
    __builtin_memcpy(&f, &b, 4);
    return f;
}

}  // namespace gpgmp
