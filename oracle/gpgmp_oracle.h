/*
 * oracle/gpgmp_oracle.h -- TEST INFRASTRUCTURE ONLY (the oracle).
 *
 * The oracle is a CPU restatement of the reference's hot path (GPGMP, the
 * simulation engine of Inchman) and a CPU replay of this project's CUDA
 * algorithms.  Only tests/, the smoke check and bench.py's CPU baseline use it;
 * the product never links it.
 *
 * Two families of functions:
 *   orc_ref_*  restate the reference's OpenCL kernels and host logic literally
 *              (Threefry-2x32 keyed per cell, one uniform per particle, C
 *              promotion rules for the kernels' double literals).  Pinned
 *              bit-exactly against the reference's own kernel sources compiled
 *              for the CPU (oracle/_ref).
 *   orc_rep_*  replay the CUDA kernels of this project (Philox-4x32 streams,
 *              binomial jump counts) with the same IEEE single-precision
 *              operations, so that seeded GPU runs compare bit for bit.
 *
 * The model description has the same memory layout as gpgmp_model_desc in
 * include/gpgmp_c.h, so one ctypes structure drives both.
 */
#ifndef GPGMP_ORACLE_H
#define GPGMP_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_reaction {
    float   rate;
    int32_t num_reactants;
    int32_t reactant_species[3];
    int32_t reactant_stoich[3];
    int32_t num_products;
    int32_t product_species[4];
    int32_t product_stoich[4];
} orc_reaction;

typedef struct orc_model {
    int32_t width, height, num_species, num_reactions;
    float   physical_length, p0, max_time, output_interval;
    int32_t max_steps;
    int32_t boundary_mask[4];   /* x-, x+, y-, y+ : 0 reflecting, 1 absorbing */
    int32_t source_mask[4];
    int32_t solver_type;        /* 0 stochastic homogeneous, 1 stochastic inhomogeneous, 2 deterministic RK4,
                                   3 stochastic inhomogeneous FPE, 4 deterministic alpha-QSS, 5/6 deterministic
                                   inhomogeneous RK4 / alpha-QSS */
    int32_t drift_method;       /* -1 field arrays, 0 homogeneous, 1 multiplicative noise, 2 OU, 3 run-time code */
    int32_t flags;              /* bit 0 nonlinear diffusivity (recompute after sweeps), bit 1 compute moments */
    float   drift_params[8];
    const float* diffusion;            /* [S] */
    const orc_reaction* reactions;     /* [R] */
    const float* field_dx;             /* [S][H][W] or NULL */
    const float* field_dy;
    const float* field_rx;
    const float* field_ry;
    const char* code_defines;          /* run-time model code (the product compiles it with NVRTC; */
    const char* drift_code;            /* the oracle takes custom hazards through orc_set_custom_hazard) */
    const char* const* custom_laws;
    const uint8_t* individual;         /* individual species (the product's lists; the oracle restates */
    int64_t individual_capacity;       /* their steps in orc_individual.c) */
    const char* new_individuals_code;
    int32_t num_fields;                /* field parameters (the product's F(f) in model code) */
    const float* field_values;
    const char* set_field_code;
    const uint8_t* reaction_mask;      /* localised reactions: [R][H][W], 0 = off in that cell; NULL: none */
} orc_model;

/* Bit r of on[r / 32] is set when reaction r may fire in cell `cell` (Reaction::
 * reactionMask, Reaction.cpp:216-235: 1 inside one of its compartments, or
 * everywhere for a reaction that has none).  At most 128 reactions. */
static inline void orc_cell_reactions(const orc_model* m, size_t cell, uint32_t on[4]) {
    on[0] = on[1] = on[2] = on[3] = 0xFFFFFFFFu;
    if (!m->reaction_mask) return;
    const size_t area = (size_t)m->width * m->height;
    on[0] = on[1] = on[2] = on[3] = 0u;
    for (int r = 0; r < m->num_reactions && r < 128; ++r)
        if (m->reaction_mask[(size_t)r * area + cell]) on[r >> 5] |= 1u << (r & 31);
}
static inline int orc_reaction_on(const uint32_t* on, int r) { return !on || ((on[r >> 5] >> (r & 31)) & 1u); }

/* ---- generators and elementary functions ---------------------------------- */
void orc_threefry2x32_20(const uint32_t ctr[2], const uint32_t key[2], uint32_t out[2]);
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
void orc_philox_fill(uint32_t k0, uint32_t k1, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t* out, int n);
void orc_logf_many(const float* x, float* y, int n);
void orc_expf_many(const float* x, float* y, int n);
void orc_sincos2pi_many(const float* u, float* s, float* c, int n);
void orc_binomial_many(uint32_t k0, uint32_t k1, const int32_t* n, const float* p, int32_t* out, int count);
void orc_poisson_many(uint32_t k0, uint32_t k1, const float* lam, int32_t* out, int count);

/* ---- reference-exact restatements -------------------------------------------- */
float orc_ref_stay_probability(const orc_model* m);
float orc_ref_cell_width(const orc_model* m);
void orc_ref_homog_diffuse(const orc_model* m, int32_t* state, int species, int32_t seed, int32_t* lost4);
/* 1: homogeneous diffusion keyed per cell and species (the reference's defect A.1,
 * identical uniforms for species diffused in the same event, corrected); 0: literal */
void orc_ref_set_species_streams(int independent);
void orc_ref_source_boundary(const orc_model* m, int32_t* state, int species, int32_t seed, int boundary, int source);
void orc_ref_gillespie(const orc_model* m, int32_t* state, int32_t seed, float deltat);
void orc_ref_inhomog_diffuse(const orc_model* m, int32_t* state, int species, int32_t seed, float dt, int sweep_y,
                             const float* dx, const float* dy, const float* rx, const float* ry, int32_t* lost4);
float orc_ref_timestep(const orc_model* m, int species, int sweep_y,
                       const float* dx, const float* dy, const float* rx, const float* ry, float* per_cell);
void orc_ref_det_diffuse(const orc_model* m, const float* in, float* out, float dt, int in_place);
void orc_ref_rk4(const orc_model* m, float* state, float deltat);
int orc_ref_solve(const orc_model* m, int32_t* state, uint32_t seed_base,
                  int32_t* snapshots, float* snap_times, int max_snapshots, int* num_snapshots, int64_t* steps);
void orc_ref_solve_many(const orc_model* m, const int32_t* init, int R, uint32_t seed_base, int32_t* finals);
int orc_ref_solve_inhom(const orc_model* m, int32_t* state, uint32_t seed_base, const float* Dx, const float* Dy,
                        const float* rx, const float* ry, int32_t* snaps, float* snap_times, int max_snaps,
                        int* nsnap, int64_t* steps);
void orc_ref_solve_many_snaps(const orc_model* m, const int32_t* init, int R, uint32_t seed_base, const float* Dx,
                              const float* Dy, const float* rx, const float* ry, int max_snaps, int32_t* snaps);

/* ---- replay of the CUDA algorithms --------------------------------------------- */
void orc_rep_init_poisson(int W, int H, int S, int R, uint32_t seed, const float* lambda_per_species, int32_t* state);
void orc_rep_ssa(const orc_model* m, int32_t* state, int R, uint32_t seed, uint32_t step_seed, float window,
                 int32_t* status);
void orc_rep_homog_diffuse(const orc_model* m, int32_t* state, int R, uint32_t seed, int species, uint32_t step_seed);
void orc_rep_inhomog_sweep(const orc_model* m, int32_t* state, int R, uint32_t seed, int species, int sweep_y,
                           uint32_t step_seed, float dt, const float* dfield, const float* rfield);
float orc_rep_timestep(const orc_model* m, int species, int sweep_y, const float* dfield, const float* rfield);
void orc_rep_diffusivity_drift(const orc_model* m, int species, float* dx, float* dy, float* rx, float* ry);
void orc_set_custom_hazard(float (*fn)(int r, const int32_t* x));
int64_t orc_rep_ind_sweep(const orc_model* m, int32_t* state, int R, uint32_t seed, int species, int dir, float dt,
                          uint32_t step_seed, uint32_t* keys, const uint32_t* ids, int64_t n, const float* props,
                          int64_t cap, float* fields);
int64_t orc_rep_ind_sort(uint32_t* keys, uint32_t* ids, int64_t n, int64_t ncells, uint32_t* killed_ids,
                         int64_t* n_killed);
float orc_rep_timestep_cells(const float* D, const float* r, int64_t n, float dx);
int orc_rep_solve(const orc_model* m, int32_t* state, int R, uint32_t seed,
                  int32_t* snapshots, float* snap_times, int max_snapshots, int* num_snapshots,
                  int64_t* steps, int32_t* status);

/* ---- deterministic solver ----------------------------------------------------- */
void orc_gs_forward_f32(int N, int steps, float F, float k, float Du, float Dv, float vx, float vy, float dt,
                        float* u, float* v);
void orc_gs_forward_f64(int N, int steps, double F, double k, double Du, double Dv, double vx, double vy, double dt,
                        double* u, double* v);
double orc_gs_loss_grad_f64(int N, int steps, double F, double k, double Du, double Dv, double vx, double vy,
                            double dt, const double* u0, const double* v0, const double* ut, const double* vt,
                            int checkpoint_every, double* grad6);
int orc_det_solve(const orc_model* m, float* state, float* snapshots, float* snap_times, int max_snapshots,
                  int* num_snapshots, int64_t* steps);
void orc_det_sweep(const orc_model* m, const float* in, float* out, int species, int sweep_y, float dt, float dx,
                   const float* D, const float* rv);
int orc_aqss_cell(const orc_model* m, float* y, float dtg, int literal);
int orc_aqss(const orc_model* m, float* state, float dtg, int literal);

/* ---- sort, scan, cell offsets, particles -------------------------------------- */
void orc_sort_pairs_u32(uint32_t* keys, uint32_t* vals, int64_t n);
void orc_exclusive_scan_u32(const uint32_t* in, uint32_t* out, int64_t n);
void orc_cell_indices_ref(const uint32_t* sorted_keys, int64_t n, int64_t ncells, uint32_t* left, uint32_t* right);
int orc_population_maintain(const uint32_t* keys, const uint32_t* ids, int64_t n, const uint32_t* start,
                            const uint32_t* count, const int32_t* goal, int64_t ncells, const uint32_t* pool,
                            int64_t npool, uint32_t seed, uint32_t step, uint32_t* keys_out, uint32_t* ids_out,
                            uint32_t* pool_out, int64_t* n_out, int64_t* npool_out);
void orc_cell_offsets(const uint32_t* sorted_keys, int64_t n, int64_t ncells, uint32_t* start, uint32_t* count);
int64_t orc_particles_run(int64_t n, float* px, float* py, uint8_t* species, int grid, float D, float vx, float vy,
                          float dt, float p_react, uint32_t seed, int step0, int nsteps);

#ifdef __cplusplus
}
#endif
#endif
