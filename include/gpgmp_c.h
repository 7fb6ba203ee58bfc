/*
 * gpgmp_c.h -- C ABI of the B200 GPGMP solvers.
 *
 * This is the drop-in boundary for Inchman's spatial simulation hot path.  The
 * reference's boundary is the abstract C++ class gpgmp::Solver
 * (exec/src/gpgmp/src/Solver.h:15-239) with the concrete HomogeneousSolver
 * (HomogeneousSolver.h:10) and InhomogeneousSolver (InhomogeneousSolver.h:11),
 * driven by DiffusionModel::oclSolve (DiffusionModel.cpp:1414-1620).  Each
 * function below names the member it replaces.
 *
 * Conventions:
 *  - every function returns GPGMP_OK (0) or a positive GPGMP_ERR_* code and never
 *    exits the process (the reference calls exit(1): Kernel.h:254-270,
 *    DiffusionModel.cpp:550-565); gpgmp_last_error() gives the message of the
 *    calling thread's last failure;
 *  - the caller owns host buffers; a handle owns its device memory;
 *  - a handle issues its work on one CUDA stream (the legacy default stream
 *    unless gpgmp_solver_set_stream is called); calls are asynchronous on that
 *    stream, the gpgmp_get_* / gpgmp_synchronize calls wait for it;
 *  - a handle is not safe to use from two host threads at once.
 *  - State layout is [realisation][species][y][x] with x fastest, the
 *    reference's per-run layout (Solver.cpp:476-482) repeated per realisation.
 */
#ifndef GPGMP_C_H
#define GPGMP_C_H
#ifndef __CUDACC_RTC__
#include <stddef.h>
#include <stdint.h>
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define GPGMP_OK 0
#define GPGMP_ERR_INVALID 1      /* bad argument or model */
#define GPGMP_ERR_CUDA 2         /* a CUDA call failed; see gpgmp_last_error() */
#define GPGMP_ERR_NOMEM 3        /* device allocation failed */
#define GPGMP_ERR_UNSUPPORTED 4  /* feature outside what this build implements */
#define GPGMP_ERR_TIMEOUT 5      /* a bounded device wait gave up (sort/scan look-back) */

/* per-realisation simulation status bits (gpgmp_get_status) */
#define GPGMP_SIM_EVENT_CAP 1    /* a cell hit the SSA event cap inside one window */
#define GPGMP_SIM_OVERFLOW 2     /* a count would have passed INT32_MAX */

/* SolverType (DiffusionModel.h:46-56); the reference's bit values 1, 2, 4, 8, 16, 32, 64
 * are numbered 0..6 here */
#define GPGMP_STOCHASTIC_HOMOGENEOUS 0             /* stochastic_homogeneous */
#define GPGMP_STOCHASTIC_INHOMOGENEOUS 1           /* stochastic_inhomogeneous */
#define GPGMP_DETERMINISTIC_RK4 2                  /* deterministic_homogeneous_RK4 */
#define GPGMP_STOCHASTIC_INHOMOGENEOUS_FPE 3       /* stochastic_inhomogeneous_fpe: FPE jump rates and time step
                                                      (StochasticInhomogeneousDriftDiffusion.cl:124-129,197-203,493-499) */
#define GPGMP_DETERMINISTIC_AQSS 4                 /* deterministic_homogeneous_aqss (Deterministic.cl:240-522) */
#define GPGMP_DETERMINISTIC_INHOMOGENEOUS_RK4 5    /* deterministic_inhomogeneous_RK4 (Deterministic.cl:71-136) */
#define GPGMP_DETERMINISTIC_INHOMOGENEOUS_AQSS 6   /* deterministic_inhomogeneous_aqss */

/* drift/diffusivity methods (DiffusionModel.cpp:319-380); FIELD takes per-cell arrays */
#define GPGMP_DRIFT_FIELD (-1)
#define GPGMP_DRIFT_HOMOGENEOUS 0          /* params: diffX, diffY, driftX, driftY */
#define GPGMP_DRIFT_MULTIPLICATIVE_NOISE 1 /* params: sigmaX, sigmaY, muX, muY */
#define GPGMP_DRIFT_ORNSTEIN_UHLENBECK 2   /* params: diffX, diffY, gammaXX, gammaXY, gammaYX, gammaYY */
#define GPGMP_DRIFT_CODE 3                 /* gpgmp_model_desc.drift_code, compiled at run time */

/* gpgmp_model_desc.flags */
#define GPGMP_FLAG_NONLINEAR 1             /* inhomogeneous, GPGMP_DRIFT_CODE: the method is evaluated again after
                                              every sweep of a species, on the state and time then, and the next
                                              time step of that direction follows (InhomogeneousSolver.cpp:303-335;
                                              stochastic solvers of one realisation) */
#define GPGMP_FLAG_COMPUTE_MOMENTS 2       /* with it, SP(i)->MeanX (the mean x of species i, helpers.cl:18-21)
                                              is computed before the first evaluation and after every x sweep */
#define GPGMP_FLAG_STOP_ON_ERROR 4         /* end a realisation's event loop once its status is set */
#define GPGMP_FLAG_LITERAL_REDIFFUSION 8   /* deterministic: repeat the stencil per due species (reference) */
#define GPGMP_FLAG_AQSS_LITERAL 16  /* alpha-QSS as the reference writes it: predictor from the current
                                       q, d with the outer step's size (Deterministic.cl:381-387) and the
                                       corrector coefficient as printed (`180.*+rtaub`, :424), instead of
                                       Mott & Oran's restart from the saved state */
#define GPGMP_FLAG_NO_INHOM_DET_REACTIONS 32 /* deterministic inhomogeneous: no reaction windows, as the
                                                reference (Solver.cpp:250-266 runs homogeneous types only) */

/* gpgmp_solver_create flags */
#define GPGMP_CREATE_SYNC_EACH_LAUNCH 1    /* wait after every launch, as Kernel.h:252-253 does */

/* A mass-action reaction (Reaction.h:31-211): hazard = rate * prod_s A_s (A_s - 1) ...
 * (Reaction.cpp:119-138, no 1/n! factor). */
typedef struct gpgmp_reaction {
    float   rate;
    int32_t num_reactants;
    int32_t reactant_species[3];
    int32_t reactant_stoich[3];
    int32_t num_products;
    int32_t product_species[4];
    int32_t product_stoich[4];
} gpgmp_reaction;

/* The model fields the hot path reads (DiffusionModel.h, Species.h:23,
 * Compartment.h:29-43; initial states are the caller's, as generateInitialStates
 * fills them host-side, DiffusionModel.cpp:568-723). */
typedef struct gpgmp_model_desc {
    int32_t width, height, num_species, num_reactions;
    float   physical_length;      /* L: cell width h = L / width */
    float   p0;                   /* redistribution fraction, default 0.1 (DiffusionModel.cpp:150) */
    float   max_time, output_interval;
    int32_t max_steps;            /* < 0: unlimited */
    int32_t boundary_mask[4];     /* x-, x+, y-, y+ : 0 reflecting, 1 absorbing (DiffusionModel.cpp:233-242) */
    int32_t source_mask[4];       /* > 0: source wall (HomogeneousSolver.cpp:210-227) */
    int32_t solver_type;          /* GPGMP_STOCHASTIC_* / GPGMP_DETERMINISTIC_* */
    int32_t drift_method;         /* GPGMP_DRIFT_* (inhomogeneous solver) */
    int32_t flags;                /* GPGMP_FLAG_* */
    float   drift_params[8];
    const float* diffusion;           /* [num_species] diffusion constants */
    const gpgmp_reaction* reactions;  /* [num_reactions] */
    const float* field_dx;            /* GPGMP_DRIFT_FIELD: [S][H][W] diffusivity x */
    const float* field_dy;            /* [S][H][W] diffusivity y */
    const float* field_rx;            /* [S][H][W] drift x */
    const float* field_ry;            /* [S][H][W] drift y */
    /* Model code compiled at run time for the device (NVRTC), as the reference
     * generates its kernels from the model (Solver.cpp:643-777, 843-905).  NULL where
     * unused.
     *  code_defines: preprocessor lines (e.g. parameter values) put before all code;
     *  drift_code:   statements of the drift/diffusivity method, GPGMP_DRIFT_CODE:
     *                they set All->DiffusivityX/Y, All->DriftX/Y of the species being
     *                computed and may read SP(i)->... of species i (State, MeanX,
     *                DiffusivityX/Y, DriftX/Y), GridX, GridY, PhysicalX, PhysicalY,
     *                PhysicalModelWidth/Height, PhysicalCellWidth/Height,
     *                GridModelWidth/Height and PhysicalSimTime; type Real = float;
     *  custom_laws:  num_reactions entries, each a C expression for the reaction's
     *                propensity in X(i) (the count of species i as float), or NULL
     *                for the mass-action hazard. */
    const char* code_defines;
    const char* drift_code;
    const char* const* custom_laws;
    /* Individual species (IndividualSolver.cpp, IndividualSolver.cl): individual[s] != 0
     * tracks the molecules of species s one by one -- a cell-sorted list of
     * individuals, each with an id and four properties (DiffusivityX, DiffusivityY,
     * DriftX, DriftY) -- in the stochastic inhomogeneous solvers.  NULL: none.
     *  individual_capacity: the most individuals one species may have over all
     *                       realisations (0: four times the initial count, at least
     *                       65,536);
     *  new_individuals_code: statements setting All->... of an individual a reaction
     *                       window created (the newIndividualsMethod; RANDOM is a
     *                       uniform draw), or NULL to keep the properties its id has.
     * With GPGMP_DRIFT_CODE the drift method runs per individual on its properties;
     * with a built-in method the individuals move with their properties as stored. */
    const uint8_t* individual;
    int64_t individual_capacity;
    const char* new_individuals_code;
    /* Field parameters (DiffusionModel.cpp:402-404, Solver.cpp:88-101,736-747): per-cell
     * values the model code reads as F(f) (field f of this cell); the caller's
     * code_defines name them (e.g. "#define conc F(0)").
     *  field_values:   [num_fields][H][W] initial values, NULL for zeros (the
     *                  reference's init scripts fill them);
     *  set_field_code: the setField method, statements run in every cell before the
     *                  diffusion of every step with deltat > 0 (updateFields,
     *                  Solver.cpp:269-272, the kernel of :583-653): F(f) and X(i) (the
     *                  count of species i as a float, written back truncated) may be
     *                  read and written; deltat and simtime are the step's.  One
     *                  realisation per solver when it is set. */
    int32_t num_fields;
    const float* field_values;
    const char* set_field_code;
    /* Localised reactions (Reaction::addCompartment / reactionMask, Reaction.h:160-189,
     * Reaction.cpp:209-235; the mask image of Solver.cpp:352-390): [num_reactions][H][W]
     * bytes, non-zero where the reaction may fire -- the union of its compartments'
     * inclusive rectangles, or every cell for a reaction with none.  The SSA hazard and
     * the deterministic right-hand side (RK4, alpha-QSS) of a reaction are zero in the
     * cells where its byte is 0 (the reference multiplies them by the mask,
     * Solver.cpp:852-854, 946-948).  NULL: every reaction everywhere. */
    const uint8_t* reaction_mask;
} gpgmp_model_desc;

typedef struct gpgmp_solver gpgmp_solver;

const char* gpgmp_last_error(void);
int gpgmp_version(void);

/* Solver(DiffusionModel&, runState, detState, SolverType, ...) -- Solver.h:33-36,
 * HomogeneousSolver.h / InhomogeneousSolver.h:28-33.  num_realisations copies of
 * the model run side by side; seed keys every random stream. */
int gpgmp_solver_create(const gpgmp_model_desc* model, int32_t num_realisations, uint32_t seed,
                        int32_t create_flags, gpgmp_solver** out);
/* ~Solver() -- Solver.cpp:174-206 */
int gpgmp_solver_destroy(gpgmp_solver* h);
/* bind the handle to a CUDA stream (cudaStream_t passed as void*) */
int gpgmp_solver_set_stream(gpgmp_solver* h, void* stream);
/* synchronizeStateBufferToDevice / FromDevice -- Solver.h:85-93, Solver.cpp:297-315.
 * Stochastic solvers take int32 counts, the deterministic solver float. */
int gpgmp_set_state(gpgmp_solver* h, const void* host_state);
int gpgmp_get_state(gpgmp_solver* h, void* host_state);
/* device-side initial state: Poisson(lambda[s]) per cell and species */
int gpgmp_init_poisson(gpgmp_solver* h, const float* lambda_per_species);
/* doReactions(Real deltat, int& seed) -- Solver.h:52, Solver.cpp:207-267 */
int gpgmp_do_reactions(gpgmp_solver* h, float deltat, int32_t* seed);
/* diffuse(int speciesIndex, Real currentTime, int& seed) -- Solver.h:80,
 * HomogeneousSolver.cpp:203-235, InhomogeneousSolver.cpp:254-427 */
int gpgmp_diffuse(gpgmp_solver* h, int32_t species, float current_time, int32_t* seed);
/* getNextDiffusionTime() -- Solver.h:68, InhomogeneousSolver.cpp:238-252 */
int gpgmp_next_diffusion_time(gpgmp_solver* h, float* out_per_species);
/* DiffusionModel::oclSolve's event loop (DiffusionModel.cpp:1414-1603) run in C++
 * over this solver.  Snapshots: the initial state, one per output interval, the
 * final state; snapshots has room for max_snapshots states (NULL to count only). */
int gpgmp_solve(gpgmp_solver* h, void* snapshots, float* snapshot_times, int32_t max_snapshots,
                int32_t* num_snapshots, int64_t* steps);
/* gpgmp_solve, calling on_dump(user, index, time) at every dump (after its snapshot
 * is copied), where the caller may read the state or the individual lists (the
 * reference's writeAllSpecies, DiffusionModel.cpp:1096-1260); a non-zero return ends
 * the run with an error. */
typedef int (*gpgmp_dump_callback)(void* user, int32_t index, float time);
int gpgmp_solve_with_callback(gpgmp_solver* h, void* snapshots, float* snapshot_times, int32_t max_snapshots,
                              int32_t* num_snapshots, int64_t* steps, gpgmp_dump_callback on_dump, void* user);
/* per-realisation GPGMP_SIM_* bits; the reference's debug error buffer
 * (Gillespie.cl:86-98, Solver.cpp:274-295) turned into a status word */
int gpgmp_get_status(gpgmp_solver* h, int32_t* status_per_realisation);
int gpgmp_synchronize(gpgmp_solver* h);
/* the device state buffer (for zero-copy views); valid until destroy */
void* gpgmp_device_state(gpgmp_solver* h);
/* computeTimestepX/Y + reduceBlocks + readback -- InhomogeneousSolver.cpp:468-500 */
int gpgmp_timesteps(gpgmp_solver* h, float* dt_x, float* dt_y);
/* Launch shapes of the stochastic kernels (the reference fixes its work-group shape,
 * Globals.h:24-28, Solver.cpp:30-33): the diffusion kernels' tile of tile_w x tile_h
 * cells (256 threads) and the SSA kernel's block of ssa_threads threads, one cell each.
 * Every draw is keyed by its cell, so the results do not depend on the shape.
 *  gpgmp_solver_launch_choices: the shapes there are (arrays of at least 8 entries,
 *                               any may be NULL);
 *  gpgmp_solver_set_launch / get_launch: choose one (GPGMP_ERR_INVALID for a shape
 *                               not among the choices) / read the current one;
 *  gpgmp_solver_autotune: times every tile shape on species 0's diffusion and every
 *                               block size on one SSA window of length `window` (<= 0:
 *                               the smallest diffusion time step) on the current state,
 *                               reps launches each, and keeps the fastest; the state,
 *                               clocks and status do not change.  ms_tiles / ms_ssa
 *                               (may be NULL) receive the mean milliseconds per launch. */
int gpgmp_solver_launch_choices(int32_t* n_tiles, int32_t* tile_w, int32_t* tile_h, int32_t* n_ssa,
                                int32_t* ssa_threads);
int gpgmp_solver_set_launch(gpgmp_solver* h, int32_t tile_w, int32_t tile_h, int32_t ssa_threads);
int gpgmp_solver_get_launch(gpgmp_solver* h, int32_t* tile_w, int32_t* tile_h, int32_t* ssa_threads);
int gpgmp_solver_autotune(gpgmp_solver* h, float window, int32_t reps, float* ms_tiles, float* ms_ssa);
/* Field parameters (Solver.h:59, :85-100): one setField pass (deltat, simtime), and
 * the fields [num_fields][H][W] to and from the host. */
int gpgmp_update_fields(gpgmp_solver* h, float deltat, float simtime);
int gpgmp_get_fields(gpgmp_solver* h, float* fields);
int gpgmp_set_fields(gpgmp_solver* h, const float* fields);
/* Individual species.  Keys are r * width * height + cell (realisation r), sorted;
 * the reference's output pairs are key | id << 32 (IndividualSolver.h:6-9,
 * getPositionList, IndividualSolver.cpp:1295-1318).
 *  gpgmp_individual_count: the individuals of species s now (all realisations);
 *  gpgmp_get_individuals:  up to capacity of them in list order -- keys, ids and the
 *                          properties [4][capacity] (any output may be NULL);
 *  gpgmp_set_individual_properties: properties [4][count] of ids first_id ..
 *                          first_id + count - 1 (the initial individuals are ids 0..
 *                          in cell order, as the reference's init scripts set them);
 *                          the next time steps follow the new properties. */
int gpgmp_individual_count(gpgmp_solver* h, int32_t species, int64_t* n);
int gpgmp_get_individuals(gpgmp_solver* h, int32_t species, uint32_t* keys, uint32_t* ids, float* props,
                          int64_t capacity, int64_t* n);
int gpgmp_set_individual_properties(gpgmp_solver* h, int32_t species, const float* props, int64_t first_id,
                                    int64_t count);


/* ---- deterministic reaction-diffusion: Gray-Scott, forward and adjoint ----------
 * The reference's deterministic solver (Deterministic.cl:17-238, driven as in
 * DiffusionModel.cpp:534-548) run on the Gray-Scott network of
 * exec/src/tests/GrayScottModel.cpp:14-60 with explicit Euler steps on a periodic
 * n x n lattice, h = 1, plus a constant drift (vx, vy) (the drift stencil of
 * Deterministic.cl:71-136).  The reference has no adjoint; gpgmp_gs_adjoint_* is the
 * hand-written discrete adjoint of the same steps.
 * Device pointers; u and v are n*n row-major arrays.  Checkpoint buffers hold
 * ceil(steps / checkpoint_every) states, each u then v. */
typedef struct gpgmp_gs_params {
    int32_t n;                  /* lattice side; a multiple of the cluster size */
    int32_t steps;
    double  F, k, Du, Dv, vx, vy, dt;
    int32_t checkpoint_every;   /* <= 0: 100 in float32, 25 in float64 */
    int32_t cluster;            /* CTAs per thread-block cluster, 0 = automatic */
    int32_t variant;            /* kernel family (float32): 0 automatic = for n = 256 the
                                   multi-cluster kernel 41 where the device holds its four clusters at
                                   once, else register-resident where the lattice allows (n 64, 128,
                                   256 on a 16-CTA cluster), else the shared-memory column walk;
                                   1 one cell per iteration; 2 shared-memory column walk;
                                   3 register-resident; 10 + w register-resident with w warps per
                                   CTA; 40 + i multi-cluster (n = 256; clusters, ghost rows):
                                   i = 0 (2, 8), 1 (4, 8), 2 (4, 16), 3 (8, 8), 4 (8, 16),
                                   5 (4, 32), 6 (2, 32), a CUDA error where the device cannot hold
                                   all its clusters at once.  Every float32 family gives the same
                                   bits.  float64 always uses 0 / 1 (column walk / per cell).  The
                                   adjoint runs the multi-cluster adjoint under 40 + i (the same
                                   lambda bits); under 0, where the forward is multi-cluster, it
                                   recomputes the segments on two clusters (40) and runs the
                                   four-cluster adjoint beside it.  The batched forward treats
                                   40 + i as 0. */
} gpgmp_gs_params;

/* bytes of the checkpoint buffer and of the adjoint's work buffer */
int gpgmp_gs_buffer_sizes(const gpgmp_gs_params* p, int32_t elem_bytes, size_t* checkpoint_bytes,
                          size_t* work_bytes);
int gpgmp_gs_forward_f32(const gpgmp_gs_params* p, const float* u0, const float* v0, float* u, float* v,
                         float* checkpoints, void* stream);
int gpgmp_gs_forward_f64(const gpgmp_gs_params* p, const double* u0, const double* v0, double* u, double* v,
                         double* checkpoints, void* stream);
/* lam_u/lam_v: dL/du_N, dL/dv_N in; grad_u0/grad_v0: dL/du_0, dL/dv_0 out;
 * grad6 (device, 6 doubles): dL/d(F, k, Du, Dv, vx, vy), overwritten. */
int gpgmp_gs_adjoint_f32(const gpgmp_gs_params* p, const float* checkpoints, const float* lam_u, const float* lam_v,
                         float* grad_u0, float* grad_v0, double* grad6, void* work, void* stream);
int gpgmp_gs_adjoint_f64(const gpgmp_gs_params* p, const double* checkpoints, const double* lam_u,
                         const double* lam_v, double* grad_u0, double* grad_v0, double* grad6, void* work,
                         void* stream);
/* batch independent float32 lattices in one launch, one 16-CTA cluster each (on a B200
 * seven or eight run at once, gpgmp_gs_batch_capacity): u0, v0, u, v are [batch][n][n]; member_params (host, may be NULL
 * = all use p) holds per member F, k, Du, Dv, vx, vy; n, steps and dt are p's.  No
 * checkpoints.  Each member's result is bit-identical to its own gpgmp_gs_forward_f32.
 * No counterpart in the reference (one model per run). */
int gpgmp_gs_forward_batch_f32(const gpgmp_gs_params* p, int32_t batch, const double* member_params,
                               const float* u0, const float* v0, float* u, float* v, void* stream);
/* how many lattices of side n gpgmp_gs_forward_batch_f32 runs at the same time on the
 * current device (its 16-CTA clusters that are resident at once) */
int gpgmp_gs_batch_capacity(int32_t n, int32_t* lattices);
/* the float32 kernel family (gpgmp_gs_params.variant) that variant 0 resolves to for an
 * n x n lattice, with (drift != 0) or without drift, on the current device */
int gpgmp_gs_auto_variant(int32_t n, int32_t drift, int32_t* variant);
/* Status of the forward kernels on the current device: *flags != 0 if a bounded wait
 * inside a register-resident forward solve gave up since the last call (that solve's
 * output is NaN).  Synchronises the device and clears the flags.  No counterpart in
 * the reference (its kernels have no waits). */
int gpgmp_gs_status(int32_t* flags);
/* Host buffers in and out: copies (u0, v0) to the device, runs the forward solve,
 * copies (u, v) back.  Its device buffers come from a memory pool per device that the
 * library keeps (freed memory stays mapped for the next call, until the process exits). */
int gpgmp_gs_forward_host(const gpgmp_gs_params* p, const float* u0, const float* v0, float* u, float* v);
/* Host buffers: loss L = sum (u_N - ut)^2 + (v_N - vt)^2 and its gradient with
 * respect to (F, k, Du, Dv, vx, vy) by the adjoint. */
int gpgmp_gs_loss_grad_host(const gpgmp_gs_params* p, const float* u0, const float* v0, const float* ut,
                            const float* vt, double* loss, double* grad6);

/* ---- individual particles: exclusive scan, radix sort, cell offsets -------------
 * The reference sorts each individual species' (cell, id) keys with a stable LSD
 * radix sort (IndividualSolver::sortSpecies / radixSortStep / scanExclusive,
 * IndividualSolver.cpp:673-808) and derives cell index ranges
 * (IndividualSolver::computeCellIndices, IndividualSolver.cpp:1083-1098,
 * kernel IndividualSolver.cl:564-619).  Device pointers; the caller passes a
 * scratch buffer of at least the queried size.  The calls are asynchronous on
 * `stream`; a look-back wait that exceeded its iteration limit is reported by
 * gpgmp_scratch_status (kind 0: scan scratch, 1: sort scratch) as GPGMP_ERR_TIMEOUT. */
int gpgmp_scan_scratch_bytes(int64_t n, size_t* bytes);
/* out[i] = in[0] + ... + in[i-1] (mod 2^32); out[0] = 0 */
int gpgmp_exclusive_scan_u32(const uint32_t* in, uint32_t* out, int64_t n, void* scratch, size_t scratch_bytes,
                             void* stream);
/* the sort's scratch size depends on n only: one buffer serves every key_bits */
int gpgmp_sort_scratch_bytes(int64_t n, int32_t key_bits, size_t* bytes);
/* stable sort of (key, value) by the low key_bits bits of key; n < 2^30; in and out
 * must not overlap */
int gpgmp_sort_pairs_u32(const uint32_t* keys_in, const uint32_t* vals_in, uint32_t* keys_out, uint32_t* vals_out,
                         int64_t n, int32_t key_bits, void* scratch, size_t scratch_bytes, void* stream);
/* count[c] = #keys == c, start[c] = exclusive scan of count (scratch: scan of ncells) */
int gpgmp_cell_offsets(const uint32_t* sorted_keys, int64_t n, int64_t ncells, uint32_t* start, uint32_t* count,
                       void* scratch, size_t scratch_bytes, void* stream);
/* the reference's cell index ranges: left = start, right = start + count - 1
 * (= start for an empty cell, the index of the next particle) */
int gpgmp_cell_indices(const uint32_t* start, const uint32_t* count, int64_t ncells, uint32_t* left, uint32_t* right,
                       void* stream);
int gpgmp_scratch_status(const void* scratch, int32_t kind, int64_t n, int32_t key_bits, int32_t* status);

/* ---- individual particles: population bookkeeping -------------------------------
 * IndividualSolver::maintainPopulation (IndividualSolver.cpp:458-671,
 * IndividualSolver.cl:1017-1882, doc/source/individual.rst).  After a reaction window
 * changed the per-cell counts goal[c], the cell-sorted list (keys = cell index, ids)
 * with its cell_start / cell_count (gpgmp_cell_offsets) is rebuilt so that cell c
 * holds goal[c] individuals: a cell's surplus is removed, chosen uniformly without
 * replacement by a random stream keyed by (seed, step, cell), and the removed ids are
 * put at the front of the new pool in list order, followed by the unused old pool;
 * a cell's missing individuals take ids from the front of the old pool, in cell
 * order, and come first in their cell, before its survivors (in their old order).
 * Outputs: keys_out / ids_out (n_active_out entries, at most capacity_out), pool_out
 * (n_pool_out ids, at most pool_capacity), start_out (optional, ncells entries: the
 * new cell starts; the new counts are goal).  Device pointers; returns after the
 * work is done (the totals are read back, into a 64-byte pinned host buffer that the
 * calling thread's first call allocates).  GPGMP_ERR_INVALID when the pool has
 * fewer free ids than births or an output is too small. */
int gpgmp_population_scratch_bytes(int64_t n_active, int64_t ncells, size_t* bytes);
int gpgmp_population_maintain(const uint32_t* keys, const uint32_t* ids, int64_t n_active,
                              const uint32_t* cell_start, const uint32_t* cell_count, const int32_t* goal,
                              int64_t ncells, const uint32_t* pool, int64_t n_pool, uint32_t seed, uint32_t step,
                              uint32_t* keys_out, uint32_t* ids_out, int64_t capacity_out, uint32_t* pool_out,
                              int64_t pool_capacity, uint32_t* start_out, int64_t* n_active_out,
                              int64_t* n_pool_out, void* scratch, size_t scratch_bytes, void* stream);
/* gpgmp_exclusive_scan_u32 for callers that may not allocate device memory: code
 * whose device memory is owned and accounted by another allocator (a framework's
 * memory pool), or that cannot take cudaMalloc's implicit synchronisation or its
 * failure in the middle of a time loop.  No counterpart in the reference.  The
 * scratch is a fixed 32 KiB device array inside the library, so n is at most
 * 2^26 (67,108,864) values; larger n is rejected with GPGMP_ERR_INVALID.  The first
 * call on each device looks the array up (cudaGetSymbolAddress) with that device
 * current; make that first call before any stream capture.  Every call on a device
 * shares the one array: calls whose kernels overlap on the GPU (other streams, other
 * host threads) race and must be serialised by the caller.  The looked-up address is
 * kept for the life of the process: do not use this entry point across a
 * cudaDeviceReset of that device.  Allocates nothing.  Like the scan above it returns
 * before the kernel ends, so a look-back wait that gave up is reported by
 * gpgmp_exclusive_scan_u32_noalloc_status, not by the return code. */
int gpgmp_exclusive_scan_u32_noalloc(const uint32_t* in, uint32_t* out, int64_t n, void* stream);
/* Waits for `stream`, then sets *status to GPGMP_ERR_TIMEOUT if the last
 * gpgmp_exclusive_scan_u32_noalloc on this device gave up a look-back wait (its output
 * is then wrong), else GPGMP_OK.  The next no-allocation scan clears the record, so
 * call this before it.  Allocates nothing. */
int gpgmp_exclusive_scan_u32_noalloc_status(void* stream, int32_t* status);

/* ---- individual particles on the lattice: move, bin, react, compact ---------------
 * The reference's individual solver (IndividualSolver.cpp:416-712, 458-671) moves
 * (cell, id) keys cell by cell, re-sorts them and keeps the population by scans and
 * compaction.  This handle keeps continuous positions and a species byte (0 = A,
 * 1 = B) per particle on a G x G lattice of unit cells; one step is a Brownian move
 * (diffusion D, drift (vx, vy), reflecting walls), binning by stable radix sort of the
 * cell index plus exclusive scan of the cell counts, in-cell A + B -> 0 (the k-th A
 * pairs with the k-th B in sorted order, each pair reacts with probability p_react)
 * and compaction of the survivors in sorted order. */
typedef struct gpgmp_particles gpgmp_particles;
int gpgmp_particles_create(int64_t capacity, int32_t grid, float D, float vx, float vy, float dt, float p_react,
                           uint32_t seed, gpgmp_particles** out);
int gpgmp_particles_destroy(gpgmp_particles* h);
int gpgmp_particles_set_stream(gpgmp_particles* h, void* stream);
/* host arrays in; step = index of the next step (keys the random streams) */
int gpgmp_particles_set(gpgmp_particles* h, const float* x, const float* y, const uint8_t* species, int64_t n,
                        int32_t step);
int gpgmp_particles_get(gpgmp_particles* h, float* x, float* y, uint8_t* species, int64_t* n);
int gpgmp_particles_step(gpgmp_particles* h, int32_t nsteps);
/* the last step's bins (host arrays, any may be NULL): start/count per cell, the sorted
 * cell keys and the sorting permutation */
int gpgmp_particles_bins(gpgmp_particles* h, uint32_t* start, uint32_t* count, uint32_t* sorted_keys,
                         uint32_t* sorted_index, int64_t* n_binned);
int gpgmp_particles_status(gpgmp_particles* h, int32_t* status);

/* ---- batched ensembles: one persistent kernel for many independent instances ------
 * Replaces running the reference's solver once per model or realisation
 * (DiffusionModel.cpp:513-532 rebuilds and reruns everything per run; every launch
 * waits, Kernel.h:252-253).  Each instance is a homogeneous stochastic model (square
 * lattice, own species, mass-action network, diffusion constants, p0, end time,
 * reflecting or absorbing walls; no source walls) whose event loop runs on the device;
 * a CTA takes instances from a queue ordered by estimated cost.  An instance gives the
 * same bits as a gpgmp_solver of the same model with seed = instance seed and
 * realisation index = instance realisation. */
typedef struct gpgmp_instance {
    int32_t width;              /* square lattice side */
    int32_t num_species, num_reactions;
    int32_t species_offset;     /* first entry of the instance in the diffusion (and lambda) array */
    int32_t reaction_offset;    /* first entry in the reaction array */
    int32_t boundary_mask[4];
    float   physical_length, p0, max_time, output_interval;
    int32_t max_steps;          /* < 0: unlimited */
    int32_t flags;              /* GPGMP_FLAG_STOP_ON_ERROR */
    uint32_t seed, realisation; /* random stream key */
    int32_t max_snapshots;
    int32_t reserved;
    int64_t state_offset;       /* first int32 of the instance's [S][W][W] counts in the state array */
    int64_t snapshot_offset;    /* first int32 of its snapshots, or -1 for none */
} gpgmp_instance;

typedef struct gpgmp_ensemble gpgmp_ensemble;
/* lambda (optional, aligned with diffusion): Poisson mean of the initial counts */
int gpgmp_ensemble_create(const gpgmp_instance* instances, int32_t n, const float* diffusion, int64_t n_diffusion,
                          const float* lambda, const gpgmp_reaction* reactions, int64_t n_reactions,
                          gpgmp_ensemble** out);
int gpgmp_ensemble_destroy(gpgmp_ensemble* h);
/* launch shape of the persistent kernel (threads 128/256/512/1024, CTAs per SM) */
int gpgmp_ensemble_configure(gpgmp_ensemble* h, int32_t threads_per_cta, int32_t ctas_per_sm);
int gpgmp_ensemble_launch_shape(gpgmp_ensemble* h, int32_t* threads, int32_t* ctas_per_sm, int32_t* grid);
/* device state: Poisson(lambda) initial counts for every instance */
int gpgmp_ensemble_init_poisson(gpgmp_ensemble* h, int32_t* state, void* stream);
/* runs every instance to its end time (device state in place, device snapshots
 * optional); captured as a CUDA graph on first use, replayed afterwards */
int gpgmp_ensemble_run(gpgmp_ensemble* h, int32_t* state, int32_t* snapshots, void* stream);
/* waits for the device; per-instance status bits and event-loop steps; snapshot
 * times of the instances with snapshots, concatenated */
int gpgmp_ensemble_results(gpgmp_ensemble* h, int32_t* status, int64_t* steps, float* snapshot_times);

#ifdef __cplusplus
}
#endif
#endif
