/*
 * oracle/ref/ref_driver.c -- TEST INFRASTRUCTURE ONLY (the reference checker).
 *
 * Runs the reference's kernels, compiled unchanged from their .cl sources by
 * ref_homog.c / ref_inhomog.c / ref_det.c, over every work-item of an NDRange in
 * order, the way the reference host enqueues them (HomogeneousSolver.cpp:203-235,
 * InhomogeneousSolver.cpp:254-427).  Each entry point is one enqueue.
 */
#include <stdio.h>
#include <stdlib.h>
#include "cl_shim.h"

size_t shim_gid[2], shim_gsize[2], shim_lid[2], shim_lsize[2], shim_group[2], shim_ngroups[2];
size_t GridModelWidth, GridModelHeight, NumReactions, NumSpecies;
Real PhysicalModelWidth, PhysicalModelHeight, PhysicalCellWidth, PhysicalCellHeight, StayProbability;
int BoundaryMaskX1, BoundaryMaskX2, BoundaryMaskY1, BoundaryMaskY2;

void homogeneous_stochastic_diffuse(int *d_state, int4 *d_lostParticles, int seed, int speciesIndex);
void homogeneous_stochastic_updateState(int *d_state, int4 *d_lostParticles, int speciesIndex);
void homogeneous_stochastic_source_boundary(int *d_state, int seed, int speciesIndex, int boundary, int source);
void inhomogeneous_diffuseX(int *d_state, float4 *tp, int4 *lost, int seed, int speciesIndex, Real dt, Real *err,
                            Real *rx, Real *ry, Real *Dx, Real *Dy);
void inhomogeneous_diffuseY(int *d_state, float4 *tp, int4 *lost, int seed, int speciesIndex, Real dt, Real *err,
                            Real *rx, Real *ry, Real *Dx, Real *Dy);
void inhomogeneous_updateStateX(int *d_state, int4 *lost, int speciesIndex);
void inhomogeneous_updateStateY(int *d_state, int4 *lost, int speciesIndex);
void inhomogeneous_computeIndividualTimestepX(Real *ts, Real *minBlock, Real *Dx, Real *Dy, Real *rx, Real *ry,
                                              float4 *tp, int speciesIndex, Real simTime, Real *err, Real *s_local);
void inhomogeneous_computeIndividualTimestepY(Real *ts, Real *minBlock, Real *Dx, Real *Dy, Real *rx, Real *ry,
                                              float4 *tp, int speciesIndex, Real simTime, Real *err, Real *s_local);
void homogeneous_deterministic_diffuse(Real *d_state, Real dtdiff, Real *_physicalDiffusionConstants);

/* the header prints every Real with std::scientific (Solver.cpp:451, :505-509) */
static float printed(double v) {
    char b[64];
    snprintf(b, sizeof b, "%e", v);
    return strtof(b, NULL);
}

void gref_set_model(int W, int H, int S, float L, float p0, const int *bmask) {
    GridModelWidth = (size_t)W;
    GridModelHeight = (size_t)H;
    NumSpecies = (size_t)S;
    NumReactions = 0;
    PhysicalModelWidth = printed(L);
    PhysicalModelHeight = printed(L);
    PhysicalCellWidth = printed(L / (float)W);
    PhysicalCellHeight = printed(L / (float)H);
    StayProbability = printed(1. - p0);
    BoundaryMaskX1 = bmask[0];
    BoundaryMaskX2 = bmask[1];
    BoundaryMaskY1 = bmask[2];
    BoundaryMaskY2 = bmask[3];
}

static void set_item(size_t x, size_t y, size_t W, size_t H, size_t lx, size_t ly) {
    shim_gid[0] = x; shim_gid[1] = y;
    shim_gsize[0] = W; shim_gsize[1] = H;
    shim_lsize[0] = lx; shim_lsize[1] = ly;
    shim_lid[0] = x % lx; shim_lid[1] = y % ly;
    shim_group[0] = x / lx; shim_group[1] = y / ly;
    shim_ngroups[0] = W / lx; shim_ngroups[1] = H / ly;
}

#define FOR_ITEMS(LX, LY) for (size_t y = 0; y < GridModelHeight; ++y) for (size_t x = 0; x < GridModelWidth; ++x) \
    if ((set_item(x, y, GridModelWidth, GridModelHeight, (LX), (LY))), 1)

void gref_homog_diffuse(int *state, int *lost4, int seed, int species) {
    FOR_ITEMS(1, 1) homogeneous_stochastic_diffuse(state, (int4 *)lost4, seed, species);
    FOR_ITEMS(1, 1) homogeneous_stochastic_updateState(state, (int4 *)lost4, species);
}

void gref_source_boundary(int *state, int seed, int species, int boundary, int source) {
    for (size_t d = 0; d < GridModelWidth; ++d) {
        set_item(d, 0, GridModelWidth, 1, 1, 1);
        homogeneous_stochastic_source_boundary(state, seed, species, boundary, source);
    }
}

void gref_inhomog_diffuse(int *state, float *Dx, float *Dy, float *rx, float *ry, int *lost4,
                          int seed, int species, float dt, int sweep_y) {
    float err[64] = {0};
    if (!sweep_y) {
        FOR_ITEMS(1, 1) inhomogeneous_diffuseX(state, NULL, (int4 *)lost4, seed, species, dt, err, rx, ry, Dx, Dy);
        FOR_ITEMS(1, 1) inhomogeneous_updateStateX(state, (int4 *)lost4, species);
    } else {
        FOR_ITEMS(1, 1) inhomogeneous_diffuseY(state, NULL, (int4 *)lost4, seed, species, dt, err, rx, ry, Dx, Dy);
        FOR_ITEMS(1, 1) inhomogeneous_updateStateY(state, (int4 *)lost4, species);
    }
}

/* local size 1: each work-group's minimum is its one cell's time step */
void gref_timestep_cells(float *Dx, float *Dy, float *rx, float *ry, int species, int sweep_y, float *per_cell) {
    float err[64] = {0}, s_local[4];
    FOR_ITEMS(1, 1) {
        if (!sweep_y)
            inhomogeneous_computeIndividualTimestepX(NULL, per_cell, Dx, Dy, rx, ry, NULL, species, 0.f, err, s_local);
        else
            inhomogeneous_computeIndividualTimestepY(NULL, per_cell, Dx, Dy, rx, ry, NULL, species, 0.f, err, s_local);
    }
}

void gref_det_diffuse_inplace(float *state, float *D, float dt) {
    FOR_ITEMS(1, 1) homogeneous_deterministic_diffuse(state, dt, D);
}

/* the vendored Random123 generators themselves (cl_include/Random123/threefry.h:733,
 * philox.h:326), for pinning the oracle's restatements */
#include <Random123/philox.h>
void gref_threefry2x32(const unsigned *ctr, const unsigned *key, unsigned *out) {
    threefry2x32_ctr_t c = {{ctr[0], ctr[1]}};
    threefry2x32_key_t k = {{key[0], key[1]}};
    threefry2x32_ctr_t r = threefry2x32(c, k);
    out[0] = r.v[0]; out[1] = r.v[1];
}
void gref_philox4x32(const unsigned *ctr, const unsigned *key, unsigned *out) {
    philox4x32_ctr_t c = {{ctr[0], ctr[1], ctr[2], ctr[3]}};
    philox4x32_key_t k = {{key[0], key[1]}};
    philox4x32_ctr_t r = philox4x32(c, k);
    for (int i = 0; i < 4; ++i) out[i] = r.v[i];
}
