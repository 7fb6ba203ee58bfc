// C++ host runtime of the B200 solvers behind the C ABI of include/gpgmp_c.h.
//
// gpgmp_solver mirrors gpgmp::Solver and its two subclasses
// (exec/src/gpgmp/src/Solver.h:15-239, HomogeneousSolver.cpp:79-235,
// InhomogeneousSolver.cpp:7-503): the host keeps the per-species diffusion
// clocks exactly as the reference does, in float, and launches one kernel per
// reaction window / diffusion sweep covering every realisation.  Nothing waits
// for the device unless the caller asks for results (or for the reference's
// finish-after-every-launch behaviour, GPGMP_CREATE_SYNC_EACH_LAUNCH).
#include <cstring>
#include <cstdio>
#include <cmath>
#include <string>
#include <vector>
#include <algorithm>
#include <cuda_runtime.h>
#include "kernels.h"
#include "host_common.h"
#include "jit.h"
#include "individual.h"

using namespace gpgmp;

struct gpgmp_solver {
    gpgmp_model_desc m{};
    std::vector<float> diffusion;
    std::vector<gpgmp_reaction> reactions;
    int R = 1;
    uint32_t seed = 0;
    int create_flags = 0;
    cudaStream_t stream = nullptr;
    GridDesc g{};
    size_t area = 0;
    bool deterministic = false, inhom = false;
    bool aqss = false;      // alpha-QSS reaction windows instead of RK4
    bool fpe = false;       // stochastic_inhomogeneous_fpe jump rates
    int ts_kind = 0;        // time step formula of the inhomogeneous solvers (TimestepKind)
    // model code compiled at run time (jit.h): parameter defines, drift method,
    // per-reaction custom propensity laws ("" = mass action)
    std::string code_defines, drift_code;
    std::vector<std::string> custom_laws;
    JitFunction jit_ssa = nullptr, jit_drift = nullptr;
    // stochastic state: two buffers, per-species current index
    int32_t* d_buf[2] = {nullptr, nullptr};
    std::vector<int> cur;
    // deterministic state: whole-state ping-pong
    float* d_fbuf[2] = {nullptr, nullptr};
    int fcur = 0;
    gpgmp_reaction* d_reactions = nullptr;
    uint32_t* d_rmask = nullptr;      // localised reactions: [words][area] bits (GridDesc::rmask), or NULL
    int32_t* d_status = nullptr;
    float* d_diff = nullptr;
    float *d_Dx = nullptr, *d_Dy = nullptr, *d_rx = nullptr, *d_ry = nullptr;
    uint32_t* d_minkey = nullptr;
    float* d_lambda = nullptr;
    void* d_stage = nullptr;          // gather buffer for snapshots / readback
    // diffusion clocks (HomogeneousSolver.h m_dt / m_nextDiffusionTime,
    // InhomogeneousSolver.h m_nextDiffusionTimeX/Y, m_smallestDtX/Y, m_diffusionDtX/Y)
    std::vector<float> dt, next;
    std::vector<float> nextX, nextY, smallX, smallY, ddX, ddY;
    float pi = 0.f, pmove = 0.f, h = 1.f, det_dt = 0.f, stay = 0.f;
    // individual species (individual.h): one list per flagged species
    std::vector<uint8_t> is_ind;
    std::vector<IndList> ind;           // indexed by species (species == -1: not individual)
    IndKernels ind_k;
    std::string newind_code;
    long long ind_cap = 0;
    float sim_time = 0.f;               // the time of the last diffusion event (the methods' PhysicalSimTime)
    // nonlinear drift methods (GPGMP_FLAG_NONLINEAR / _COMPUTE_MOMENTS)
    bool nonlinear = false, moments = false;
    float* d_meanx = nullptr;               // [S]
    unsigned long long* d_msums = nullptr;  // [2]
    // field parameters (Solver.cpp:88-101) and the setField method
    int nfields = 0;
    float* d_fields = nullptr;              // [F][area]
    std::string set_field_code;
    JitFunction jit_fields = nullptr;
};

namespace {

bool is_inhom_type(int t) {
    return t == GPGMP_STOCHASTIC_INHOMOGENEOUS || t == GPGMP_STOCHASTIC_INHOMOGENEOUS_FPE ||
           t == GPGMP_DETERMINISTIC_INHOMOGENEOUS_RK4 || t == GPGMP_DETERMINISTIC_INHOMOGENEOUS_AQSS;
}

#define CK(expr)                                                                       \
    do {                                                                               \
        cudaError_t e_ = (expr);                                                       \
        if (e_ != cudaSuccess) return set_error(GPGMP_ERR_CUDA, "%s: %s", #expr, cudaGetErrorString(e_)); \
    } while (0)

int after_launch(gpgmp_solver* h, cudaError_t e) {
    if (e != cudaSuccess) return set_error(GPGMP_ERR_CUDA, "launch: %s", cudaGetErrorString(e));
    if (h->create_flags & GPGMP_CREATE_SYNC_EACH_LAUNCH) {
        e = cudaStreamSynchronize(h->stream);
        if (e != cudaSuccess) return set_error(GPGMP_ERR_CUDA, "sync: %s", cudaGetErrorString(e));
    }
    return GPGMP_OK;
}

Planes planes_of(gpgmp_solver* h) {
    Planes p{};
    for (int s = 0; s < h->g.S; ++s) p.p[s] = h->d_buf[h->cur[s]];
    return p;
}

// Gathers the per-species planes into one contiguous [R][S][area] device buffer.
int gather_state(gpgmp_solver* h, void* dst) {
    const size_t plane_bytes = h->area * sizeof(int32_t);
    bool uniform = true;
    for (int s = 0; s < h->g.S; ++s) uniform = uniform && h->cur[s] == h->cur[0];
    if (uniform) {
        CK(cudaMemcpyAsync(dst, h->d_buf[h->cur[0]], plane_bytes * h->g.S * h->R, cudaMemcpyDeviceToDevice, h->stream));
        return GPGMP_OK;
    }
    CK(cudaMemcpy2DAsync(dst, plane_bytes, h->d_buf[0], plane_bytes, plane_bytes, (size_t)h->g.S * h->R,
                         cudaMemcpyDeviceToDevice, h->stream));
    for (int s = 0; s < h->g.S; ++s) {
        if (h->cur[s] == 0) continue;
        // species s of every realisation: R planes with a pitch of S planes
        CK(cudaMemcpy2DAsync((char*)dst + s * plane_bytes, plane_bytes * h->g.S,
                             (const char*)h->d_buf[1] + s * plane_bytes, plane_bytes * h->g.S, plane_bytes, h->R,
                             cudaMemcpyDeviceToDevice, h->stream));
    }
    return GPGMP_OK;
}

// Makes buffer 0 hold every plane (so the state is one contiguous array).
int normalize(gpgmp_solver* h) {
    if (h->deterministic) {
        if (h->fcur == 1) {
            CK(cudaMemcpyAsync(h->d_fbuf[0], h->d_fbuf[1], h->area * h->g.S * h->R * sizeof(float),
                               cudaMemcpyDeviceToDevice, h->stream));
            h->fcur = 0;
        }
        return GPGMP_OK;
    }
    const size_t plane_bytes = h->area * sizeof(int32_t);
    for (int s = 0; s < h->g.S; ++s) {
        if (h->cur[s] == 0) continue;
        CK(cudaMemcpy2DAsync((char*)h->d_buf[0] + s * plane_bytes, plane_bytes * h->g.S,
                             (const char*)h->d_buf[1] + s * plane_bytes, plane_bytes * h->g.S, plane_bytes, h->R,
                             cudaMemcpyDeviceToDevice, h->stream));
        h->cur[s] = 0;
    }
    return GPGMP_OK;
}

void free_all(gpgmp_solver* h) {
    void* ptrs[] = {h->d_buf[0], h->d_buf[1], h->d_fbuf[0], h->d_fbuf[1], h->d_reactions, h->d_status, h->d_diff,
                    h->d_Dx, h->d_Dy, h->d_rx, h->d_ry, h->d_minkey, h->d_lambda, h->d_stage, h->d_meanx,
                    h->d_msums, h->d_fields, h->d_rmask};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    for (IndList& l : h->ind) ind_free(l);
}

int validate(const gpgmp_model_desc* m, int R) {
    if (!m) return set_error(GPGMP_ERR_INVALID, "model is NULL");
    if (m->width <= 0 || m->height <= 0) return set_error(GPGMP_ERR_INVALID, "grid %dx%d", m->width, m->height);
    if (m->num_species <= 0 || m->num_species > kMaxSpecies)
        return set_error(GPGMP_ERR_INVALID, "num_species %d outside 1..%d", m->num_species, kMaxSpecies);
    if (m->num_reactions < 0 || m->num_reactions > 128)
        return set_error(GPGMP_ERR_INVALID, "num_reactions %d outside 0..128", m->num_reactions);
    if (m->num_reactions > 0 && !m->reactions) return set_error(GPGMP_ERR_INVALID, "reactions is NULL");
    if (!m->diffusion) return set_error(GPGMP_ERR_INVALID, "diffusion is NULL");
    if (R <= 0) return set_error(GPGMP_ERR_INVALID, "num_realisations %d", R);
    if ((int64_t)m->width * m->height > (int64_t)1 << 30) return set_error(GPGMP_ERR_INVALID, "grid too large");
    for (int i = 0; i < m->num_reactions; ++i) {
        const gpgmp_reaction& r = m->reactions[i];
        if (r.num_reactants < 0 || r.num_reactants > 3 || r.num_products < 0 || r.num_products > 4)
            return set_error(GPGMP_ERR_INVALID, "reaction %d: bad reactant/product count", i);
        for (int j = 0; j < r.num_reactants; ++j)
            if (r.reactant_species[j] < 0 || r.reactant_species[j] >= m->num_species || r.reactant_stoich[j] < 0)
                return set_error(GPGMP_ERR_INVALID, "reaction %d: bad reactant %d", i, j);
        for (int j = 0; j < r.num_products; ++j)
            if (r.product_species[j] < 0 || r.product_species[j] >= m->num_species || r.product_stoich[j] < 0)
                return set_error(GPGMP_ERR_INVALID, "reaction %d: bad product %d", i, j);
    }
    if (m->solver_type < 0 || m->solver_type > 6) return set_error(GPGMP_ERR_UNSUPPORTED, "solver_type %d", m->solver_type);
    if (is_inhom_type(m->solver_type)) {
        if (m->drift_method == GPGMP_DRIFT_FIELD &&
            (!m->field_dx || !m->field_dy || !m->field_rx || !m->field_ry))
            return set_error(GPGMP_ERR_INVALID, "field drift method needs all four field arrays");
        if (m->drift_method < GPGMP_DRIFT_FIELD || m->drift_method > GPGMP_DRIFT_CODE)
            return set_error(GPGMP_ERR_UNSUPPORTED, "drift_method %d", m->drift_method);
        if (m->drift_method == GPGMP_DRIFT_CODE && !m->drift_code)
            return set_error(GPGMP_ERR_INVALID, "GPGMP_DRIFT_CODE needs drift_code");
        if ((m->flags & (GPGMP_FLAG_NONLINEAR | GPGMP_FLAG_COMPUTE_MOMENTS)) && m->drift_method == GPGMP_DRIFT_CODE) {
            if (m->solver_type != GPGMP_STOCHASTIC_INHOMOGENEOUS && m->solver_type != GPGMP_STOCHASTIC_INHOMOGENEOUS_FPE)
                return set_error(GPGMP_ERR_UNSUPPORTED, "nonlinear drift methods with a deterministic solver");
            if (R != 1)
                return set_error(GPGMP_ERR_UNSUPPORTED,
                                 "a nonlinear drift method needs one realisation per solver (its fields follow the state)");
        }
    }
    if (m->num_fields < 0) return set_error(GPGMP_ERR_INVALID, "num_fields %d", m->num_fields);
    if (m->set_field_code && m->set_field_code[0]) {
        if (m->num_fields <= 0) return set_error(GPGMP_ERR_INVALID, "set_field_code without fields");
        const int ty = m->solver_type;
        if (ty != GPGMP_STOCHASTIC_HOMOGENEOUS && ty != GPGMP_STOCHASTIC_INHOMOGENEOUS &&
            ty != GPGMP_STOCHASTIC_INHOMOGENEOUS_FPE)
            return set_error(GPGMP_ERR_UNSUPPORTED, "a setField method with a deterministic solver");
        if (R != 1) return set_error(GPGMP_ERR_UNSUPPORTED, "a setField method needs one realisation per solver");
    }
    if (m->individual) {
        bool any = false;
        for (int s = 0; s < m->num_species; ++s) any = any || m->individual[s];
        if (any && m->solver_type != GPGMP_STOCHASTIC_INHOMOGENEOUS && m->solver_type != GPGMP_STOCHASTIC_INHOMOGENEOUS_FPE)
            return set_error(GPGMP_ERR_UNSUPPORTED, "individual species need a stochastic inhomogeneous solver");
        if (any && (int64_t)m->width * m->height * R >= ((int64_t)1 << 31))
            return set_error(GPGMP_ERR_INVALID, "individual species: realisations x cells must stay below 2^31");
        if (m->individual_capacity < 0) return set_error(GPGMP_ERR_INVALID, "individual_capacity < 0");
    }
    return GPGMP_OK;
}

IndArgs ind_args(gpgmp_solver* h, int species, int dir, float dt, uint32_t step_seed) {
    IndArgs a{};
    a.W = h->g.W;
    a.H = h->g.H;
    a.S = h->g.S;
    a.R = h->R;
    a.species = species;
    a.dir = dir;
    a.L = h->m.physical_length;
    a.dx = h->m.physical_length / (float)(dir == 0 ? h->m.width : h->m.height);
    a.dt = dt;
    a.sim_time = h->sim_time;
    for (int b = 0; b < 4; ++b) a.bmask[b] = h->m.boundary_mask[b];
    a.seed = h->seed;
    a.step_seed = step_seed;
    Planes p = planes_of(h);
    for (int s = 0; s < h->g.S; ++s) a.planes[s] = p.p[s];
    return a;
}

// The smallest time step over every cell of every realisation from a species'
// individual fields (computeIndividualTimestepX/Y on the fields that
// computeDiffusionConstants wrote, InhomogeneousSolver.cpp:468-500).
int ind_timestep(gpgmp_solver* h, const IndList& l, int dir, float* out) {
    const float dx = h->m.physical_length / (float)(dir == 0 ? h->m.width : h->m.height);
    const float* D = l.fields + (dir == 0 ? 0 : l.ncells);
    const float* r = l.fields + (dir == 0 ? 2 : 3) * l.ncells;
    uint32_t key = 0;
    CK(launch_timestep((int)l.ncells, D, r, dx, h->d_minkey, h->stream, h->ts_kind, h->stay));
    CK(cudaMemcpyAsync(&key, h->d_minkey, 4, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    *out = key_to_float(key);
    return GPGMP_OK;
}

// (Re)builds the individual lists from the state (the caller set it) and takes the
// first time steps from them (InhomogeneousSolver.cpp:190-211 for individual species).
int ind_refresh(gpgmp_solver* h, const int32_t* host_state) {
    if (h->ind.empty()) return GPGMP_OK;
    const long long ncells = (long long)h->area * h->R;
    for (int s = 0; s < h->g.S; ++s) {
        IndList& l = h->ind[s];
        if (l.species < 0) continue;
        long long cap = h->ind_cap;
        if (cap <= 0) {
            long long n0 = 0;
            if (host_state) {
                for (int r = 0; r < h->R; ++r) {
                    const int32_t* p = host_state + ((size_t)r * h->g.S + s) * h->area;
                    for (size_t c = 0; c < h->area; ++c) n0 += p[c] > 0 ? p[c] : 0;
                }
            } else {
                std::vector<int32_t> st((size_t)h->area * h->g.S * h->R);
                int rc = gather_state(h, h->d_stage);
                if (rc) return rc;
                CK(cudaMemcpyAsync(st.data(), h->d_stage, st.size() * sizeof(int32_t), cudaMemcpyDeviceToHost,
                                   h->stream));
                CK(cudaStreamSynchronize(h->stream));
                for (int r = 0; r < h->R; ++r)
                    for (size_t c = 0; c < h->area; ++c) n0 += st[((size_t)r * h->g.S + s) * h->area + c];
            }
            cap = 4 * n0 > 65536 ? 4 * n0 : 65536;
            if (cap >= ((long long)1 << 31)) cap = ((long long)1 << 31) - 1;
        }
        if (l.cap != cap || l.ncells != ncells || !l.keys[0]) {
            bool may_leave = false;
            for (int b = 0; b < 4; ++b) may_leave = may_leave || h->m.boundary_mask[b] != 0;
            int rc = ind_alloc(l, s, cap, ncells, may_leave);
            if (rc) return rc;
        }
        int rc = ind_build(l, ind_args(h, s, 0, 0.f, 0u), h->ind_k, h->stream);
        if (rc) return rc;
        rc = ind_timestep(h, l, 0, &h->smallX[s]);
        if (rc) return rc;
        rc = ind_timestep(h, l, 1, &h->smallY[s]);
        if (rc) return rc;
        h->ddX[s] = h->smallX[s];
        h->ddY[s] = h->smallY[s];
        h->nextX[s] = h->smallX[s];
        h->nextY[s] = h->smallY[s];
        h->next[s] = h->nextX[s] < h->nextY[s] ? h->nextX[s] : h->nextY[s];
    }
    return GPGMP_OK;
}

// InhomogeneousSolver.cpp:164-212: diffusivity/drift per species, then the first
// time steps (computeTimestepX/Y read back one float each; the formula depends on
// the solver type).
int inhom_init(gpgmp_solver* h) {
    const size_t n = h->area * h->g.S;
    if (h->m.drift_method == GPGMP_DRIFT_CODE) {
        // the reference's generated inhomogeneous_computeDiffusionConstants_forSpecies_<id>
        // kernels, run species after species on fields that start at zero
        CK(cudaMemsetAsync(h->d_Dx, 0, n * sizeof(float), h->stream));
        CK(cudaMemsetAsync(h->d_Dy, 0, n * sizeof(float), h->stream));
        CK(cudaMemsetAsync(h->d_rx, 0, n * sizeof(float), h->stream));
        CK(cudaMemsetAsync(h->d_ry, 0, n * sizeof(float), h->stream));
        if (!h->jit_drift) {
            int rc = jit_drift_kernel(h->code_defines, h->drift_code, &h->jit_drift);
            if (rc) return rc;
        }
        Planes planes{};
        if (!h->deterministic) planes = planes_of(h);
        if (h->moments)   // the reference computes the moments of every species first (:168-185)
            for (int s = 0; s < h->g.S; ++s)
                CK(launch_moments(planes.p[s] + (size_t)s * h->area, h->m.width, h->m.height, h->m.physical_length,
                                  h->d_msums, h->d_meanx + s, h->stream));
        for (int s = 0; s < h->g.S; ++s)
            CK(launch_drift_jit(h->jit_drift, h->g, s, h->m.physical_length, 0.f, h->d_Dx, h->d_Dy, h->d_rx, h->d_ry,
                                h->deterministic ? nullptr : &planes, h->moments ? h->d_meanx : nullptr, h->d_fields,
                                h->stream));
    } else if (h->m.drift_method == GPGMP_DRIFT_FIELD) {
        CK(cudaMemcpyAsync(h->d_Dx, h->m.field_dx, n * sizeof(float), cudaMemcpyHostToDevice, h->stream));
        CK(cudaMemcpyAsync(h->d_Dy, h->m.field_dy, n * sizeof(float), cudaMemcpyHostToDevice, h->stream));
        CK(cudaMemcpyAsync(h->d_rx, h->m.field_rx, n * sizeof(float), cudaMemcpyHostToDevice, h->stream));
        CK(cudaMemcpyAsync(h->d_ry, h->m.field_ry, n * sizeof(float), cudaMemcpyHostToDevice, h->stream));
    } else {
        for (int s = 0; s < h->g.S; ++s)
            CK(launch_diffusivity_drift(h->g, s, h->m.drift_method, h->m.drift_params, h->m.physical_length, h->d_Dx,
                                        h->d_Dy, h->d_rx, h->d_ry, h->stream));
    }
    const float dx = h->m.physical_length / (float)h->m.width;
    for (int s = 0; s < h->g.S; ++s) {
        uint32_t key[2];
        CK(launch_timestep((int)h->area, h->d_Dx + s * h->area, h->d_rx + s * h->area, dx, h->d_minkey, h->stream,
                           h->ts_kind, h->stay));
        CK(cudaMemcpyAsync(&key[0], h->d_minkey, 4, cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        CK(launch_timestep((int)h->area, h->d_Dy + s * h->area, h->d_ry + s * h->area, dx, h->d_minkey, h->stream,
                           h->ts_kind, h->stay));
        CK(cudaMemcpyAsync(&key[1], h->d_minkey, 4, cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        h->smallX[s] = key_to_float(key[0]);
        h->smallY[s] = key_to_float(key[1]);
        h->ddX[s] = h->smallX[s];
        h->ddY[s] = h->smallY[s];
        h->nextX[s] = h->smallX[s];
        h->nextY[s] = h->smallY[s];
    }
    return GPGMP_OK;
}

// A nonlinear drift method after a sweep of species i in direction dir
// (InhomogeneousSolver.cpp:288-335): the moments after an x sweep, the method on the
// state and time now, the smallest time step of that direction.
int nonlinear_update(gpgmp_solver* h, int i, int dir, float t) {
    if (!h->nonlinear) return GPGMP_OK;
    Planes planes = planes_of(h);
    if (h->moments && dir == 0)
        CK(launch_moments(planes.p[i] + (size_t)i * h->area, h->m.width, h->m.height, h->m.physical_length, h->d_msums,
                          h->d_meanx + i, h->stream));
    CK(launch_drift_jit(h->jit_drift, h->g, i, h->m.physical_length, t, h->d_Dx, h->d_Dy, h->d_rx, h->d_ry, &planes,
                        h->moments ? h->d_meanx : nullptr, h->d_fields, h->stream));
    const float dx = h->m.physical_length / (float)h->m.width;
    uint32_t key = 0;
    CK(launch_timestep((int)h->area, (dir == 0 ? h->d_Dx : h->d_Dy) + (size_t)i * h->area,
                       (dir == 0 ? h->d_rx : h->d_ry) + (size_t)i * h->area, dx, h->d_minkey, h->stream, h->ts_kind,
                       h->stay));
    CK(cudaMemcpyAsync(&key, h->d_minkey, 4, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    (dir == 0 ? h->smallX[i] : h->smallY[i]) = key_to_float(key);
    return GPGMP_OK;
}

// A drift method in code may read the counts (SP(i)->State): like the reference's
// solver constructor, evaluate it on the initial state, i.e. again once the caller
// has set the state.
int refresh_code_fields(gpgmp_solver* h) {
    if (!h->inhom || h->m.drift_method != GPGMP_DRIFT_CODE) return GPGMP_OK;
    int rc = inhom_init(h);
    if (rc) return rc;
    for (int i = 0; i < h->g.S; ++i) h->next[i] = h->nextX[i] < h->nextY[i] ? h->nextX[i] : h->nextY[i];
    return GPGMP_OK;
}

}  // namespace

extern "C" {

int gpgmp_version(void) { return 100; }

int gpgmp_solver_create(const gpgmp_model_desc* model, int32_t num_realisations, uint32_t seed, int32_t create_flags,
                        gpgmp_solver** out) {
    if (!out) return set_error(GPGMP_ERR_INVALID, "out is NULL");
    *out = nullptr;
    int rc = validate(model, num_realisations);
    if (rc) return rc;
    auto* h = new gpgmp_solver();
    h->m = *model;
    h->R = num_realisations;
    h->seed = seed;
    h->create_flags = create_flags;
    h->diffusion.assign(model->diffusion, model->diffusion + model->num_species);
    if (model->num_reactions > 0) h->reactions.assign(model->reactions, model->reactions + model->num_reactions);
    h->m.diffusion = h->diffusion.data();
    h->m.reactions = h->reactions.empty() ? nullptr : h->reactions.data();
    if (model->code_defines) h->code_defines = model->code_defines;
    if (model->drift_code) h->drift_code = model->drift_code;
    bool custom = false;
    if (model->custom_laws) {
        h->custom_laws.assign(model->num_reactions, std::string());
        for (int r = 0; r < model->num_reactions; ++r)
            if (model->custom_laws[r] && model->custom_laws[r][0]) {
                h->custom_laws[r] = model->custom_laws[r];
                custom = true;
            }
    }
    h->is_ind.assign(model->num_species, 0);
    bool any_ind = false;
    if (model->individual)
        for (int s = 0; s < model->num_species; ++s) {
            h->is_ind[s] = model->individual[s] ? 1 : 0;
            any_ind = any_ind || h->is_ind[s];
        }
    if (model->new_individuals_code) h->newind_code = model->new_individuals_code;
    h->ind_cap = model->individual_capacity;
    h->m.code_defines = h->m.drift_code = nullptr;
    h->m.custom_laws = nullptr;
    h->m.individual = nullptr;
    h->m.new_individuals_code = nullptr;
    h->m.field_values = nullptr;
    h->m.set_field_code = nullptr;
    h->m.reaction_mask = nullptr;
    if (any_ind) {
        h->ind.resize(model->num_species);
        for (int s = 0; s < model->num_species; ++s) h->ind[s].species = h->is_ind[s] ? s : -1;
        const bool code = model->drift_method == GPGMP_DRIFT_CODE && !h->drift_code.empty();
        if (code || !h->newind_code.empty()) {
            // the reference compiles its individual kernels with the model's methods
            // (IndividualSolver.cpp:188-330)
            int rc2 = jit_ind_kernels(h->code_defines, code ? h->drift_code : std::string(), h->newind_code,
                                      model->num_species, &h->ind_k);
            if (rc2) {
                delete h;
                return rc2;
            }
            if (!code) h->ind_k.sweep = h->ind_k.fields = nullptr;   // properties as stored
        }
    }
    const int ty = model->solver_type;
    h->deterministic = ty == GPGMP_DETERMINISTIC_RK4 || ty == GPGMP_DETERMINISTIC_AQSS ||
                       ty == GPGMP_DETERMINISTIC_INHOMOGENEOUS_RK4 || ty == GPGMP_DETERMINISTIC_INHOMOGENEOUS_AQSS;
    h->inhom = is_inhom_type(ty);
    h->aqss = ty == GPGMP_DETERMINISTIC_AQSS || ty == GPGMP_DETERMINISTIC_INHOMOGENEOUS_AQSS;
    h->fpe = ty == GPGMP_STOCHASTIC_INHOMOGENEOUS_FPE;
    h->ts_kind = h->deterministic ? 2 : (h->fpe ? 1 : 0);
    if (custom && h->deterministic) {
        delete h;
        return set_error(GPGMP_ERR_UNSUPPORTED, "custom propensity laws with a deterministic solver");
    }
    if (custom) {
        // the reference generates its Gillespie kernel from the laws (Solver.cpp:843-905)
        int rc2 = jit_ssa_kernel(h->code_defines, h->custom_laws, &h->jit_ssa);
        if (rc2) {
            delete h;
            return rc2;
        }
    }
    h->g.W = model->width;
    h->g.H = model->height;
    h->g.S = model->num_species;
    h->g.R = num_realisations;
    for (int i = 0; i < 4; ++i) h->g.bmask[i] = model->boundary_mask[i];
    h->area = (size_t)model->width * model->height;
    h->cur.assign(h->g.S, 0);
    const int S = h->g.S;
    const size_t n = h->area * S * (size_t)h->R;
    h->h = model->physical_length / (float)model->width;
    auto fail = [&](int code) {
        free_all(h);
        delete h;
        return code;
    };
#define CKC(expr)                                                                          \
    do {                                                                                   \
        cudaError_t e_ = (expr);                                                           \
        if (e_ != cudaSuccess) {                                                           \
            int c_ = set_error(e_ == cudaErrorMemoryAllocation ? GPGMP_ERR_NOMEM : GPGMP_ERR_CUDA, "%s: %s", #expr, \
                               cudaGetErrorString(e_));                                    \
            return fail(c_);                                                               \
        }                                                                                  \
    } while (0)
    if (h->deterministic) {
        CKC(cudaMalloc(&h->d_fbuf[0], n * sizeof(float)));
        CKC(cudaMalloc(&h->d_fbuf[1], n * sizeof(float)));
        CKC(cudaMemset(h->d_fbuf[0], 0, n * sizeof(float)));
        CKC(cudaMalloc(&h->d_stage, n * sizeof(float)));
    } else {
        CKC(cudaMalloc(&h->d_buf[0], n * sizeof(int32_t)));
        CKC(cudaMalloc(&h->d_buf[1], n * sizeof(int32_t)));
        CKC(cudaMemset(h->d_buf[0], 0, n * sizeof(int32_t)));
        CKC(cudaMalloc(&h->d_stage, n * sizeof(int32_t)));
    }
    CKC(cudaMalloc(&h->d_status, sizeof(int32_t) * h->R));
    CKC(cudaMemset(h->d_status, 0, sizeof(int32_t) * h->R));
    CKC(cudaMalloc(&h->d_diff, sizeof(float) * S));
    CKC(cudaMemcpy(h->d_diff, h->diffusion.data(), sizeof(float) * S, cudaMemcpyHostToDevice));
    CKC(cudaMalloc(&h->d_lambda, sizeof(float) * S));
    if (model->num_fields > 0) {
        const size_t fb = sizeof(float) * h->area * (size_t)model->num_fields;
        h->nfields = model->num_fields;
        CKC(cudaMalloc(&h->d_fields, fb));
        if (model->field_values) CKC(cudaMemcpy(h->d_fields, model->field_values, fb, cudaMemcpyHostToDevice));
        else CKC(cudaMemset(h->d_fields, 0, fb));
    }
    if (model->set_field_code && model->set_field_code[0]) {
        h->set_field_code = model->set_field_code;
        int rc2 = jit_field_kernel(h->code_defines, h->set_field_code, &h->jit_fields);
        if (rc2) return fail(rc2);
    }
    if (!h->reactions.empty()) {
        CKC(cudaMalloc(&h->d_reactions, sizeof(gpgmp_reaction) * h->reactions.size()));
        CKC(cudaMemcpy(h->d_reactions, h->reactions.data(), sizeof(gpgmp_reaction) * h->reactions.size(),
                       cudaMemcpyHostToDevice));
    }
    if (model->reaction_mask && !h->reactions.empty()) {
        // localised reactions (Solver.cpp:352-390 builds the same mask as a float image):
        // one bit per reaction and cell, 32 reactions to a word, words cell-contiguous
        const int nr = (int)h->reactions.size(), words = (nr + 31) / 32;
        std::vector<uint32_t> bits((size_t)words * h->area, 0u);
        bool all_on = true;
        for (int r = 0; r < nr; ++r)
            for (size_t c = 0; c < h->area; ++c) {
                const bool on = model->reaction_mask[(size_t)r * h->area + c] != 0;
                all_on = all_on && on;
                if (on) bits[(size_t)(r >> 5) * h->area + c] |= 1u << (r & 31);
            }
        if (!all_on) {    // a mask that is on everywhere changes nothing: no masked kernels
            CKC(cudaMalloc(&h->d_rmask, sizeof(uint32_t) * bits.size()));
            CKC(cudaMemcpy(h->d_rmask, bits.data(), sizeof(uint32_t) * bits.size(), cudaMemcpyHostToDevice));
            h->g.rmask = h->d_rmask;
            h->g.rmask_words = words;
        }
    }
    // stay probability and jump probability as the reference's header computes them
    const float stay = (float)(1.0 - (double)model->p0);
    h->stay = stay;
    h->pi = (float)((1.0 - (double)stay) / 6.0);
    h->pmove = h->pi * 4.0f;
    h->dt.assign(S, 0.f);
    h->next.assign(S, 0.f);
    if (h->deterministic && !h->inhom) {
        // HomogeneousSolver.cpp:168-192: one common step, the smallest over species
        float dtd = 0.f;
        for (int i = 0; i < S; ++i) {
            float d = h->diffusion[i] > 0 ? (float)1e-2f * h->h * h->h / (4.f * h->diffusion[i]) : model->max_time;
            if (i == 0 || d < dtd) dtd = d;
        }
        h->det_dt = dtd;
        for (int i = 0; i < S; ++i) { h->dt[i] = dtd; h->next[i] = dtd; }
    } else if (!h->inhom) {
        // HomogeneousSolver.cpp:154-166: dt_i = p0 / (2 * 3) * h^2 / D_i
        for (int i = 0; i < S; ++i) {
            h->dt[i] = h->diffusion[i] > 0 ? model->p0 / ((float)2. * 3) * h->h * h->h / h->diffusion[i]
                                           : model->max_time;
            h->next[i] = h->dt[i];
        }
    } else {
        const size_t nf = h->area * S;
        CKC(cudaMalloc(&h->d_Dx, nf * sizeof(float)));
        CKC(cudaMalloc(&h->d_Dy, nf * sizeof(float)));
        CKC(cudaMalloc(&h->d_rx, nf * sizeof(float)));
        CKC(cudaMalloc(&h->d_ry, nf * sizeof(float)));
        CKC(cudaMalloc(&h->d_minkey, sizeof(uint32_t)));
        h->nonlinear = (model->flags & GPGMP_FLAG_NONLINEAR) && model->drift_method == GPGMP_DRIFT_CODE;
        h->moments = (model->flags & GPGMP_FLAG_COMPUTE_MOMENTS) && model->drift_method == GPGMP_DRIFT_CODE &&
                     !h->deterministic;
        CKC(cudaMalloc(&h->d_meanx, sizeof(float) * S));
        CKC(cudaMemset(h->d_meanx, 0, sizeof(float) * S));
        CKC(cudaMalloc(&h->d_msums, 2 * sizeof(unsigned long long)));
        h->nextX.assign(S, 0.f); h->nextY.assign(S, 0.f);
        h->smallX.assign(S, 0.f); h->smallY.assign(S, 0.f);
        h->ddX.assign(S, 0.f); h->ddY.assign(S, 0.f);
        int rc2 = inhom_init(h);
        if (rc2) return fail(rc2);
        for (int i = 0; i < S; ++i) h->next[i] = h->nextX[i] < h->nextY[i] ? h->nextX[i] : h->nextY[i];
    }
    // the model's field arrays are the caller's; they were copied above if used
    h->m.field_dx = h->m.field_dy = h->m.field_rx = h->m.field_ry = nullptr;
#undef CKC
    *out = h;
    return GPGMP_OK;
}

int gpgmp_solver_destroy(gpgmp_solver* h) {
    if (!h) return GPGMP_OK;
    cudaStreamSynchronize(h->stream);
    free_all(h);
    delete h;
    return GPGMP_OK;
}

int gpgmp_solver_set_stream(gpgmp_solver* h, void* stream) {
    if (!h) return set_error(GPGMP_ERR_INVALID, "handle is NULL");
    h->stream = (cudaStream_t)stream;
    return GPGMP_OK;
}

int gpgmp_set_state(gpgmp_solver* h, const void* host) {
    if (!h || !host) return set_error(GPGMP_ERR_INVALID, "NULL argument");
    const size_t n = h->area * h->g.S * (size_t)h->R;
    if (h->deterministic) {
        CK(cudaMemcpyAsync(h->d_fbuf[0], host, n * sizeof(float), cudaMemcpyHostToDevice, h->stream));
        h->fcur = 0;
    } else {
        CK(cudaMemcpyAsync(h->d_buf[0], host, n * sizeof(int32_t), cudaMemcpyHostToDevice, h->stream));
        std::fill(h->cur.begin(), h->cur.end(), 0);
    }
    CK(cudaStreamSynchronize(h->stream));
    int rc = refresh_code_fields(h);
    if (rc) return rc;
    return h->deterministic ? GPGMP_OK : ind_refresh(h, (const int32_t*)host);
}

int gpgmp_get_state(gpgmp_solver* h, void* host) {
    if (!h || !host) return set_error(GPGMP_ERR_INVALID, "NULL argument");
    const size_t n = h->area * h->g.S * (size_t)h->R;
    if (h->deterministic) {
        CK(cudaMemcpyAsync(host, h->d_fbuf[h->fcur], n * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
    } else {
        int rc = gather_state(h, h->d_stage);
        if (rc) return rc;
        CK(cudaMemcpyAsync(host, h->d_stage, n * sizeof(int32_t), cudaMemcpyDeviceToHost, h->stream));
    }
    CK(cudaStreamSynchronize(h->stream));
    return GPGMP_OK;
}

void* gpgmp_device_state(gpgmp_solver* h) {
    if (!h) return nullptr;
    if (normalize(h)) return nullptr;
    return h->deterministic ? (void*)h->d_fbuf[0] : (void*)h->d_buf[0];
}

int gpgmp_init_poisson(gpgmp_solver* h, const float* lambda) {
    if (!h || !lambda) return set_error(GPGMP_ERR_INVALID, "NULL argument");
    if (h->deterministic) return set_error(GPGMP_ERR_UNSUPPORTED, "Poisson initial state is for stochastic solvers");
    CK(cudaMemcpyAsync(h->d_lambda, lambda, sizeof(float) * h->g.S, cudaMemcpyHostToDevice, h->stream));
    std::fill(h->cur.begin(), h->cur.end(), 0);
    int rc = after_launch(h, launch_init_poisson(h->g, planes_of(h), h->seed, h->d_lambda, h->stream));
    if (rc) return rc;
    rc = refresh_code_fields(h);
    if (rc) return rc;
    return ind_refresh(h, nullptr);
}

int gpgmp_do_reactions(gpgmp_solver* h, float deltat, int32_t* seed) {
    if (!h || !seed) return set_error(GPGMP_ERR_INVALID, "NULL argument");
    if (h->deterministic) {
        if (h->inhom && (h->m.flags & GPGMP_FLAG_NO_INHOM_DET_REACTIONS)) return GPGMP_OK;
        if (h->aqss)
            return after_launch(h, launch_aqss(h->g, h->d_fbuf[h->fcur], h->d_reactions, (int)h->reactions.size(),
                                               deltat, (h->m.flags & GPGMP_FLAG_AQSS_LITERAL) ? 1 : 0,
                                               h->d_status, h->stream));
        return after_launch(h, launch_rk4(h->g, h->d_fbuf[h->fcur], h->d_reactions, (int)h->reactions.size(), deltat,
                                          h->stream));
    }
    int rc = after_launch(h, h->jit_ssa ? launch_ssa_jit(h->jit_ssa, h->g, planes_of(h), h->d_reactions,
                                                         (int)h->reactions.size(), h->seed, (uint32_t)*seed, deltat,
                                                         h->d_status, h->stream)
                                        : launch_ssa(h->g, planes_of(h), h->d_reactions, (int)h->reactions.size(),
                                                     h->seed, (uint32_t)*seed, deltat, h->d_status, h->stream));
    (*seed)++;
    if (rc) return rc;
    // the individual species follow the new counts (Solver.cpp:240-247: one seed each)
    for (IndList& l : h->ind) {
        if (l.species < 0) continue;
        rc = ind_maintain(l, ind_args(h, l.species, 0, 0.f, (uint32_t)*seed), h->ind_k, h->stream);
        (*seed)++;
        if (rc) return rc;
    }
    return GPGMP_OK;
}

int gpgmp_diffuse(gpgmp_solver* h, int32_t i, float t, int32_t* seed) {
    if (!h || !seed) return set_error(GPGMP_ERR_INVALID, "NULL argument");
    if (i < 0 || i >= h->g.S) return set_error(GPGMP_ERR_INVALID, "species %d", i);
    const size_t plane_stride = 0;
    (void)plane_stride;
    if (h->deterministic && !h->inhom) {
        int rc = after_launch(h, launch_det_diffuse(h->g, h->d_fbuf[h->fcur], h->d_fbuf[1 - h->fcur], h->d_diff,
                                                    h->dt[i], h->h * h->h, h->stream));
        h->fcur ^= 1;
        h->next[i] += h->dt[i];
        return rc;
    }
    if (!h->inhom) {
        const int c = h->cur[i];
        int rc = after_launch(h, launch_homog_diffuse(h->g, h->d_buf[c], h->d_buf[1 - c], i, h->seed, (uint32_t)*seed,
                                                      h->pmove, h->stream));
        if (rc) return rc;
        h->cur[i] ^= 1;
        int32_t* base = h->d_buf[h->cur[i]];
        const int* sm = h->m.source_mask;
        // HomogeneousSolver.cpp:212-227 (wall 0 takes its count from source_mask[1])
        const int counts[4] = {sm[1], sm[1], sm[2], sm[3]};
        for (int b = 0; b < 4; ++b) {
            if (sm[b] > 0) {
                rc = after_launch(h, launch_source(h->g, base, i, h->seed, (uint32_t)*seed, b, counts[b], h->pi,
                                                   h->stream));
                if (rc) return rc;
            }
        }
        h->next[i] += h->dt[i];
        return GPGMP_OK;
    }
    const float dxw = h->m.physical_length / (float)h->m.width;
    const float dyw = h->m.physical_length / (float)h->m.height;
    if (h->deterministic) {
        // InhomogeneousSolver::diffuse, deterministic branch (:282-287, :374-378): the
        // sweeps take no random numbers, so the seed does not advance
        for (int dir = 0; dir < 2; ++dir) {
            float& nxt = dir == 0 ? h->nextX[i] : h->nextY[i];
            if (!(nxt <= t)) continue;
            int rc = after_launch(h, launch_det_sweep(h->g, h->d_fbuf[h->fcur], h->d_fbuf[1 - h->fcur], i, dir,
                                                      dir == 0 ? h->d_Dx : h->d_Dy, dir == 0 ? h->d_rx : h->d_ry,
                                                      dir == 0 ? h->ddX[i] : h->ddY[i], dir == 0 ? dxw : dyw,
                                                      h->stream));
            if (rc) return rc;
            h->fcur ^= 1;
            nxt += dir == 0 ? h->smallX[i] : h->smallY[i];
            (dir == 0 ? h->ddX[i] : h->ddY[i]) = dir == 0 ? h->smallX[i] : h->smallY[i];
        }
        h->next[i] = h->nextX[i] < h->nextY[i] ? h->nextX[i] : h->nextY[i];
        return GPGMP_OK;
    }
    if (!h->ind.empty() && h->ind[i].species >= 0) {
        // InhomogeneousSolver::diffuse for an individual species (:264-269, :303-335):
        // move the individuals, then new fields and a new time step of that direction
        // Both sweeps go out before the host waits: the y sweep takes the time step
        // known before this call, so the x sweep's results are read with its own.
        // A sweep that fails to go out stops the loop, but a sweep already out is still
        // booked (its departures and time step), so the list stays consistent.
        h->sim_time = t;
        bool swept[2] = {false, false};
        int rc_launch = GPGMP_OK;
        for (int dir = 0; dir < 2; ++dir) {
            if (!((dir == 0 ? h->nextX[i] : h->nextY[i]) <= t)) continue;
            const float dd = dir == 0 ? h->ddX[i] : h->ddY[i];
            const float dxd = h->m.physical_length / (float)(dir == 0 ? h->m.width : h->m.height);
            rc_launch = ind_sweep(h->ind[i], ind_args(h, i, dir, dd, (uint32_t)*seed), h->ind_k, dxd, h->ts_kind,
                                  h->stay, dir, h->stream);
            if (rc_launch) break;
            (*seed)++;
            swept[dir] = true;
        }
        if (swept[0] || swept[1]) {
            cudaError_t e = cudaStreamSynchronize(h->stream);
            if (e != cudaSuccess)
                return rc_launch ? rc_launch
                                 : set_error(GPGMP_ERR_CUDA, "individual sweeps: %s", cudaGetErrorString(e));
        }
        for (int dir = 0; dir < 2; ++dir) {
            if (!swept[dir]) continue;
            float& small = dir == 0 ? h->smallX[i] : h->smallY[i];
            small = ind_sweep_result(h->ind[i], dir);
            (dir == 0 ? h->nextX[i] : h->nextY[i]) += small;
            (dir == 0 ? h->ddX[i] : h->ddY[i]) = small;
        }
        h->next[i] = h->nextX[i] < h->nextY[i] ? h->nextX[i] : h->nextY[i];
        return rc_launch;
    }
    if (h->nextX[i] <= t) {
        const int c = h->cur[i];
        int rc = after_launch(h, launch_sweep(h->g, h->d_buf[c], h->d_buf[1 - c], i, 0, h->seed, (uint32_t)*seed,
                                              h->d_Dx, h->d_rx, h->ddX[i], dxw, h->stream, h->fpe ? 1 : 0));
        if (rc) return rc;
        h->cur[i] ^= 1;
        (*seed)++;
        rc = nonlinear_update(h, i, 0, t);
        if (rc) return rc;
        h->nextX[i] += h->smallX[i];
        h->ddX[i] = h->smallX[i];
    }
    if (h->nextY[i] <= t) {
        const int c = h->cur[i];
        int rc = after_launch(h, launch_sweep(h->g, h->d_buf[c], h->d_buf[1 - c], i, 1, h->seed, (uint32_t)*seed,
                                              h->d_Dy, h->d_ry, h->ddY[i], dyw, h->stream, h->fpe ? 1 : 0));
        if (rc) return rc;
        h->cur[i] ^= 1;
        (*seed)++;
        rc = nonlinear_update(h, i, 1, t);
        if (rc) return rc;
        h->nextY[i] += h->smallY[i];
        h->ddY[i] = h->smallY[i];
    }
    h->next[i] = h->nextX[i] < h->nextY[i] ? h->nextX[i] : h->nextY[i];
    return GPGMP_OK;
}

int gpgmp_next_diffusion_time(gpgmp_solver* h, float* out) {
    if (!h || !out) return set_error(GPGMP_ERR_INVALID, "NULL argument");
    for (int i = 0; i < h->g.S; ++i) out[i] = h->next[i];
    return GPGMP_OK;
}

int gpgmp_solver_set_launch(gpgmp_solver* h, int32_t tile_w, int32_t tile_h, int32_t ssa_threads) {
    if (!h) return set_error(GPGMP_ERR_INVALID, "handle is NULL");
    int tile = -1, ssa = -1;
    for (int i = 0; i < kNumDiffusionTiles; ++i) {
        int w, hh;
        diffusion_tile_shape(i, &w, &hh);
        if (w == tile_w && hh == tile_h) tile = i;
    }
    for (int i = 0; i < kNumSsaThreadChoices; ++i)
        if (ssa_thread_choice(i) == ssa_threads) ssa = i;
    if (tile < 0) return set_error(GPGMP_ERR_INVALID, "no diffusion tile of %d x %d cells", tile_w, tile_h);
    if (ssa < 0) return set_error(GPGMP_ERR_INVALID, "no SSA block of %d threads", ssa_threads);
    h->g.tile = tile;
    h->g.ssa_threads = ssa;
    return GPGMP_OK;
}

int gpgmp_solver_get_launch(gpgmp_solver* h, int32_t* tile_w, int32_t* tile_h, int32_t* ssa_threads) {
    if (!h) return set_error(GPGMP_ERR_INVALID, "handle is NULL");
    int w, hh;
    diffusion_tile_shape(h->g.tile, &w, &hh);
    if (tile_w) *tile_w = w;
    if (tile_h) *tile_h = hh;
    if (ssa_threads) *ssa_threads = ssa_thread_choice(h->g.ssa_threads);
    return GPGMP_OK;
}

int gpgmp_solver_launch_choices(int32_t* n_tiles, int32_t* tile_w, int32_t* tile_h, int32_t* n_ssa,
                                int32_t* ssa_threads) {
    if (n_tiles) *n_tiles = kNumDiffusionTiles;
    if (n_ssa) *n_ssa = kNumSsaThreadChoices;
    for (int i = 0; i < kNumDiffusionTiles; ++i) {
        int w, hh;
        diffusion_tile_shape(i, &w, &hh);
        if (tile_w) tile_w[i] = w;
        if (tile_h) tile_h[i] = hh;
    }
    for (int i = 0; i < kNumSsaThreadChoices; ++i)
        if (ssa_threads) ssa_threads[i] = ssa_thread_choice(i);
    return GPGMP_OK;
}

// Times every diffusion tile shape on species 0's jumps (homogeneous) or x sweep
// (inhomogeneous), and every SSA block size on one reaction window of `window`, on
// the solver's current state, and keeps the fastest of each.  The kernels write only
// the spare half of the state buffers (the diffusion kernels write out of place; the
// SSA runs on a copy there) and a scratch status array, so the state, the clocks and
// the status stay as they were.
int gpgmp_solver_autotune(gpgmp_solver* h, float window, int32_t reps, float* ms_tiles, float* ms_ssa) {
    if (!h) return set_error(GPGMP_ERR_INVALID, "handle is NULL");
    if (h->deterministic) return GPGMP_OK;     // the deterministic kernels have no launch choices
    if (reps < 1) reps = 1;
    if (!(window > 0.f)) {
        window = h->m.max_time;
        for (int i = 0; i < h->g.S; ++i) {
            const float d = h->inhom ? std::min(h->smallX[i], h->smallY[i]) : h->dt[i];
            if (d > 0.f && d < window) window = d;
        }
    }
    cudaEvent_t a = nullptr, b = nullptr;
    int32_t* d_st = nullptr;
    int rc = GPGMP_OK;
    auto fail = [&](cudaError_t e, const char* what) {
        rc = set_error(GPGMP_ERR_CUDA, "autotune %s: %s", what, cudaGetErrorString(e));
    };
    cudaError_t e = cudaEventCreate(&a);
    if (e == cudaSuccess) e = cudaEventCreate(&b);
    if (e == cudaSuccess) e = cudaMalloc(&d_st, sizeof(int32_t) * (size_t)h->R);
    if (e != cudaSuccess) fail(e, "set-up");
    const GridDesc keep = h->g;
    const float dxw = h->m.physical_length / (float)h->m.width;
    const int c0 = h->cur[0];
    // one diffusion launch of tile shape i (in: species 0's current plane, out: the spare one)
    auto diffusion = [&](GridDesc& g) -> cudaError_t {
        if (!h->inhom)
            return launch_homog_diffuse(g, h->d_buf[c0], h->d_buf[1 - c0], 0, h->seed, 1u, h->pmove, h->stream);
        return launch_sweep(g, h->d_buf[c0], h->d_buf[1 - c0], 0, 0, h->seed, 1u, h->d_Dx, h->d_rx,
                            h->ddX[0] > 0.f ? h->ddX[0] : h->smallX[0], dxw, h->stream, h->fpe ? 1 : 0);
    };
    auto time_it = [&](auto&& launch, float* ms) -> cudaError_t {
        cudaError_t ee = launch();                               // warm-up (module load, caches)
        if (ee == cudaSuccess) ee = cudaEventRecord(a, h->stream);
        for (int k = 0; k < reps && ee == cudaSuccess; ++k) ee = launch();
        if (ee == cudaSuccess) ee = cudaEventRecord(b, h->stream);
        if (ee == cudaSuccess) ee = cudaEventSynchronize(b);
        if (ee == cudaSuccess) ee = cudaEventElapsedTime(ms, a, b);
        return ee;
    };
    int best_tile = keep.tile, best_ssa = keep.ssa_threads;
    float best = 0.f;
    for (int i = 0; rc == GPGMP_OK && i < kNumDiffusionTiles; ++i) {
        GridDesc g = keep;
        g.tile = i;
        float ms = 0.f;
        e = time_it([&] { return diffusion(g); }, &ms);
        if (e != cudaSuccess) { fail(e, "diffusion"); break; }
        if (ms_tiles) ms_tiles[i] = ms / reps;
        if (i == 0 || ms < best) { best = ms; best_tile = i; }
    }
    // SSA: a copy of the state in the spare buffers (every species' plane of every
    // realisation), restored before each block size so each runs the same window
    const int nreac = (int)h->reactions.size();
    if (rc == GPGMP_OK && nreac > 0 && !h->jit_ssa) {
        Planes spare{};
        for (int s = 0; s < h->g.S; ++s) spare.p[s] = h->d_buf[1 - h->cur[s]];
        const size_t plane = h->area * sizeof(int32_t);
        auto restore = [&]() -> cudaError_t {
            for (int s = 0; s < h->g.S; ++s) {
                cudaError_t ee = cudaMemcpy2DAsync((char*)spare.p[s] + s * plane, plane * h->g.S,
                                                   (const char*)h->d_buf[h->cur[s]] + s * plane, plane * h->g.S,
                                                   plane, (size_t)h->R, cudaMemcpyDeviceToDevice, h->stream);
                if (ee != cudaSuccess) return ee;
            }
            return cudaSuccess;
        };
        best = 0.f;
        for (int i = 0; i < kNumSsaThreadChoices; ++i) {
            GridDesc g = keep;
            g.ssa_threads = i;
            float ms = 0.f, total = 0.f;
            e = cudaSuccess;
            for (int k = 0; k < reps && e == cudaSuccess; ++k) {
                e = restore();
                if (e == cudaSuccess)
                    e = time_it([&] { return launch_ssa(g, spare, h->d_reactions, nreac, h->seed, 7u, window, d_st,
                                                        h->stream); }, &ms);
                total += ms;
            }
            if (e != cudaSuccess) { fail(e, "SSA"); break; }
            if (ms_ssa) ms_ssa[i] = total / reps;
            if (i == 0 || total < best) { best = total; best_ssa = i; }
        }
    }
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    if (d_st) cudaFree(d_st);
    if (rc == GPGMP_OK) {
        h->g.tile = best_tile;
        h->g.ssa_threads = best_ssa;
    }
    return rc;
}

int gpgmp_timesteps(gpgmp_solver* h, float* dtx, float* dty) {
    if (!h || !dtx || !dty) return set_error(GPGMP_ERR_INVALID, "NULL argument");
    if (!h->inhom) return set_error(GPGMP_ERR_INVALID, "time steps per direction exist for the inhomogeneous solver");
    for (int i = 0; i < h->g.S; ++i) { dtx[i] = h->smallX[i]; dty[i] = h->smallY[i]; }
    return GPGMP_OK;
}

int gpgmp_update_fields(gpgmp_solver* h, float deltat, float simtime) {
    if (!h) return set_error(GPGMP_ERR_INVALID, "handle is NULL");
    if (!h->jit_fields) return GPGMP_OK;   // no setField method
    return after_launch(h, launch_field_jit(h->jit_fields, h->g, h->m.physical_length, deltat, simtime, h->d_fields,
                                            planes_of(h), h->stream));
}

int gpgmp_get_fields(gpgmp_solver* h, float* fields) {
    if (!h || !fields) return set_error(GPGMP_ERR_INVALID, "NULL argument");
    if (h->nfields <= 0) return GPGMP_OK;
    CK(cudaMemcpyAsync(fields, h->d_fields, sizeof(float) * h->area * (size_t)h->nfields, cudaMemcpyDeviceToHost,
                       h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return GPGMP_OK;
}

int gpgmp_set_fields(gpgmp_solver* h, const float* fields) {
    if (!h || !fields) return set_error(GPGMP_ERR_INVALID, "NULL argument");
    if (h->nfields <= 0) return set_error(GPGMP_ERR_INVALID, "the model has no field parameters");
    CK(cudaMemcpyAsync(h->d_fields, fields, sizeof(float) * h->area * (size_t)h->nfields, cudaMemcpyHostToDevice,
                       h->stream));
    CK(cudaStreamSynchronize(h->stream));
    // the drift method reads the fields: like a state change, evaluate it again
    return refresh_code_fields(h);
}

int gpgmp_individual_count(gpgmp_solver* h, int32_t species, int64_t* n) {
    if (!h || !n) return set_error(GPGMP_ERR_INVALID, "NULL argument");
    if (species < 0 || species >= h->g.S || h->ind.empty() || h->ind[species].species < 0)
        return set_error(GPGMP_ERR_INVALID, "species %d is not an individual species", species);
    *n = ind_count(h->ind[species]);
    return GPGMP_OK;
}

int gpgmp_get_individuals(gpgmp_solver* h, int32_t species, uint32_t* keys, uint32_t* ids, float* props,
                          int64_t capacity, int64_t* n) {
    int rc = gpgmp_individual_count(h, species, n);
    if (rc) return rc;
    rc = ind_sort(h->ind[species], h->stream);   // the cell order (the sweeps leave it unsorted)
    if (rc) return rc;
    const IndList& l = h->ind[species];
    const long long m = l.n < capacity ? l.n : (capacity > 0 ? capacity : 0);
    if (m > 0 && keys)
        CK(cudaMemcpyAsync(keys, l.keys[l.cur], sizeof(uint32_t) * m, cudaMemcpyDeviceToHost, h->stream));
    if (m > 0 && (ids || props)) {
        std::vector<uint32_t> hid(m);
        CK(cudaMemcpyAsync(hid.data(), l.ids[l.cur], sizeof(uint32_t) * m, cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        if (ids) std::memcpy(ids, hid.data(), sizeof(uint32_t) * m);
        if (props) {
            std::vector<float> all((size_t)4 * l.cap);
            CK(cudaMemcpyAsync(all.data(), l.props, sizeof(float) * all.size(), cudaMemcpyDeviceToHost, h->stream));
            CK(cudaStreamSynchronize(h->stream));
            for (int q = 0; q < 4; ++q)
                for (long long i = 0; i < m; ++i) props[q * capacity + i] = all[(size_t)q * l.cap + hid[i]];
        }
    }
    CK(cudaStreamSynchronize(h->stream));
    return GPGMP_OK;
}

int gpgmp_set_individual_properties(gpgmp_solver* h, int32_t species, const float* props, int64_t first_id,
                                    int64_t count) {
    int64_t n = 0;
    int rc = gpgmp_individual_count(h, species, &n);
    if (rc) return rc;
    IndList& l = h->ind[species];
    if (!props || first_id < 0 || count < 0 || first_id + count > l.cap)
        return set_error(GPGMP_ERR_INVALID, "ids %lld..%lld outside the capacity %lld", (long long)first_id,
                         (long long)(first_id + count - 1), (long long)l.cap);
    for (int q = 0; q < 4; ++q)
        CK(cudaMemcpyAsync(l.props + (size_t)q * l.cap + first_id, props + (size_t)q * count, sizeof(float) * count,
                           cudaMemcpyHostToDevice, h->stream));
    // the fields and the next time steps follow the properties (as after the
    // reference's init script)
    rc = ind_fields(l, ind_args(h, species, 0, 0.f, 0u), h->ind_k, h->stream);
    if (rc) return rc;
    rc = ind_timestep(h, l, 0, &h->smallX[species]);
    if (rc) return rc;
    rc = ind_timestep(h, l, 1, &h->smallY[species]);
    if (rc) return rc;
    h->ddX[species] = h->smallX[species];
    h->ddY[species] = h->smallY[species];
    h->nextX[species] = h->sim_time + h->smallX[species];
    h->nextY[species] = h->sim_time + h->smallY[species];
    h->next[species] = h->nextX[species] < h->nextY[species] ? h->nextX[species] : h->nextY[species];
    return GPGMP_OK;
}

int gpgmp_get_status(gpgmp_solver* h, int32_t* status) {
    if (!h || !status) return set_error(GPGMP_ERR_INVALID, "NULL argument");
    CK(cudaMemcpyAsync(status, h->d_status, sizeof(int32_t) * h->R, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return GPGMP_OK;
}

int gpgmp_synchronize(gpgmp_solver* h) {
    if (!h) return set_error(GPGMP_ERR_INVALID, "handle is NULL");
    CK(cudaStreamSynchronize(h->stream));
    return GPGMP_OK;
}

// DiffusionModel::oclSolve (DiffusionModel.cpp:1414-1603).  Step n uses the
// stream seed 64 n (the reference draws boost::uniform_int + n, :1482); every
// doReactions and every inhomogeneous sweep advances it by one, as the
// reference does.  Output events take two passes of the loop (the first only
// re-arms, :1555-1571), and ties between events go to diffusion.
int gpgmp_solve(gpgmp_solver* h, void* snaps, float* snap_times, int32_t max_snaps, int32_t* nsnap, int64_t* steps) {
    return gpgmp_solve_with_callback(h, snaps, snap_times, max_snaps, nsnap, steps, nullptr, nullptr);
}

int gpgmp_solve_with_callback(gpgmp_solver* h, void* snaps, float* snap_times, int32_t max_snaps, int32_t* nsnap,
                              int64_t* steps, gpgmp_dump_callback on_dump, void* user) {
    if (!h) return set_error(GPGMP_ERR_INVALID, "handle is NULL");
    const int S = h->g.S;
    const size_t elem = h->deterministic ? sizeof(float) : sizeof(int32_t);
    const size_t block = h->area * S * (size_t)h->R * elem;
    int ns = 0;
    auto snap = [&](float t) -> int {
        if (snaps && ns < max_snaps) {
            char* dst = (char*)snaps + (size_t)ns * block;
            if (h->deterministic) {
                CK(cudaMemcpyAsync(dst, h->d_fbuf[h->fcur], block, cudaMemcpyDeviceToHost, h->stream));
            } else {
                int rc = gather_state(h, h->d_stage);
                if (rc) return rc;
                CK(cudaMemcpyAsync(dst, h->d_stage, block, cudaMemcpyDeviceToHost, h->stream));
            }
            CK(cudaStreamSynchronize(h->stream));
        }
        if (snap_times && ns < max_snaps) snap_times[ns] = t;
        if (on_dump) {
            CK(cudaStreamSynchronize(h->stream));
            if (on_dump(user, ns, t) != 0) return set_error(GPGMP_ERR_INVALID, "the dump callback failed");
        }
        ns++;
        return GPGMP_OK;
    };
    const bool stop_on_error = (h->m.flags & GPGMP_FLAG_STOP_ON_ERROR) != 0;
    std::vector<int32_t> st_host(h->R);
    int rc = snap(0.f);
    if (rc) return rc;
    float simTime = 0.f, outputLast = 0.f;
    int64_t n = 0;
    const gpgmp_model_desc& m = h->m;
    while ((m.max_steps < 0 || n < m.max_steps) && simTime < m.max_time) {
        int32_t seed = (int32_t)((uint32_t)n * 64u);
        n++;
        float mindt = h->next[0];
        int minspec = 0;
        for (int i = 1; i < S; ++i)
            if (h->next[i] < mindt) { mindt = h->next[i]; minspec = i; }
        int ev = 0;
        const float mo = outputLast + m.output_interval;
        if (mo < mindt) { mindt = mo; ev = 1; }
        const float deltat = mindt - simTime;
        if (m.num_reactions > 0) {
            rc = gpgmp_do_reactions(h, deltat, &seed);
            if (rc) return rc;
        }
        if (h->jit_fields && deltat > 0) {   // DiffusionModel.cpp:1536-1538
            rc = gpgmp_update_fields(h, deltat, simTime);
            if (rc) return rc;
        }
        if (ev == 0) {
            bool applied = false;
            for (int i = 0; i < S; ++i) {
                if (!(i == minspec || h->next[i] <= mindt)) continue;
                if (!(h->next[i] > 0)) continue;
                if (h->deterministic && !h->inhom && applied && !(m.flags & GPGMP_FLAG_LITERAL_REDIFFUSION)) {
                    h->next[i] += h->dt[i];
                    continue;
                }
                rc = gpgmp_diffuse(h, i, mindt, &seed);
                if (rc) return rc;
                applied = true;
            }
        } else if (simTime >= outputLast + m.output_interval) {
            rc = snap(mindt);
            if (rc) return rc;
            outputLast += m.output_interval;
        }
        simTime = mindt;
        if (stop_on_error && (!h->deterministic || h->aqss)) {
            rc = gpgmp_get_status(h, st_host.data());
            if (rc) return rc;
            bool any = false;
            for (int v : st_host) any = any || v != 0;
            if (any) break;
        }
    }
    rc = snap(simTime);
    if (rc) return rc;
    CK(cudaStreamSynchronize(h->stream));
    if (nsnap) *nsnap = ns;
    if (steps) *steps = n;
    return GPGMP_OK;
}

}  // extern "C"
