// Batched ensembles: thousands of independent SSA + diffusion instances (own grid
// size, species, reaction network, rates) in ONE persistent kernel.
//
// A CTA takes instances from an atomic work queue (in decreasing estimated cost,
// longest-processing-time order) and runs each one's whole event loop on the device
// -- the loop of DiffusionModel::oclSolve (DiffusionModel.cpp:1414-1603) with the
// homogeneous solver's time steps (HomogeneousSolver.cpp:154-166): SSA windows
// (Gillespie.cl:58-99) over all cells, then the lattice jumps of the due species
// (StochasticHomogeneousDiffusion.cl:8-124), snapshots at output times.  The random
// streams and every float operation are those of the wide kernels and the host loop,
// so an instance gives the same bits here as in its own gpgmp_solver (the reference's
// one-launch-per-kernel structure).  The launch (queue reset + kernel) is captured
// once in a CUDA graph and replayed.
//
// Compiled with -fmad=false.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>
#include <cuda_runtime.h>
#include "host_common.h"
#include "stoch_device.cuh"
#include "../../include/gpgmp_c.h"

using namespace gpgmp;

namespace {

struct Ctrl {
    float simTime, outputLast, mindt, window;
    int ev, minspec, stop, n;
    int nsnap;
};

struct EnsArgs {
    const gpgmp_instance* inst;
    const int32_t* order;
    int max_reactions;
    const float* diffusion;
    const gpgmp_reaction* reactions;
    int32_t* state;
    int32_t* snapshots;
    float* snap_times;       // [instance][max_snapshots] (index = snapshot_offset / block... host computes)
    int64_t* snap_time_off;  // per instance: first float of its snapshot times, or -1
    int32_t* status;
    int64_t* steps;
    int32_t* lost;           // [slot][max_area * 4]
    int64_t lost_stride;
    unsigned int* queue;
    int n_inst;
    int max_species;
};

__global__ void k_ensemble(EnsArgs A) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ gpgmp_instance s_inst;
    __shared__ Ctrl c;
    __shared__ float s_D[MAX_SPECIES], s_dt[MAX_SPECIES], s_next[MAX_SPECIES];
    __shared__ int s_item;
    const int NT = blockDim.x;
    gpgmp_reaction* rt = reinterpret_cast<gpgmp_reaction*>(smem);
    uint32_t* deps = reinterpret_cast<uint32_t*>(smem + sizeof(gpgmp_reaction) * MAX_REACTIONS);
    int* xs = reinterpret_cast<int*>(deps + 4 * MAX_REACTIONS);
    float* hs = reinterpret_cast<float*>(xs + (size_t)A.max_species * NT);
    int32_t* lost = A.lost + (int64_t)blockIdx.x * A.lost_stride;
    for (;;) {
        if (threadIdx.x == 0) s_item = (int)atomicAdd(A.queue, 1u);
        __syncthreads();
        const int item = s_item;
        if (item >= A.n_inst) break;
        const int id = A.order[item];
        if (threadIdx.x == 0) s_inst = A.inst[id];
        __syncthreads();
        const int W = s_inst.width, area = W * W, S = s_inst.num_species, R = s_inst.num_reactions;
        for (int i = threadIdx.x; i < R; i += NT) rt[i] = A.reactions[s_inst.reaction_offset + i];
        __syncthreads();
        build_deps(rt, R, deps);
        int32_t* st = A.state + s_inst.state_offset;
        const uint32_t key0 = s_inst.seed, key1 = s_inst.realisation;
        const int bm[4] = {s_inst.boundary_mask[0], s_inst.boundary_mask[1], s_inst.boundary_mask[2],
                           s_inst.boundary_mask[3]};
        if (threadIdx.x == 0) {
            // HomogeneousSolver.cpp:154-166, in float as the host does it
            const float h = s_inst.physical_length / (float)W;
            for (int i = 0; i < S; ++i) {
                const float D = A.diffusion[s_inst.species_offset + i];
                s_D[i] = D;
                s_dt[i] = D > 0 ? s_inst.p0 / ((float)2. * 3) * h * h / D : s_inst.max_time;
                s_next[i] = s_dt[i];
            }
            c.simTime = 0.f;
            c.outputLast = 0.f;
            c.n = 0;
            c.stop = 0;
            c.nsnap = 0;
        }
        __syncthreads();
        // stay and jump probabilities (as gpgmp_solver_create computes them)
        const float stay = (float)(1.0 - (double)s_inst.p0);
        const float pi = (float)((1.0 - (double)stay) / 6.0);
        const float pmove = pi * 4.0f;
        int32_t* snaps = s_inst.snapshot_offset >= 0 ? A.snapshots + s_inst.snapshot_offset : nullptr;
        float* stimes = A.snap_time_off[id] >= 0 ? A.snap_times + A.snap_time_off[id] : nullptr;
        auto snapshot = [&](float t) {
            const int k = c.nsnap;   // read by all threads before thread 0 advances it
            if (snaps && k < s_inst.max_snapshots) {
                int32_t* dst = snaps + (int64_t)k * S * area;
                for (int i = threadIdx.x; i < S * area; i += NT) dst[i] = st[i];
                if (threadIdx.x == 0 && stimes) stimes[k] = t;
            }
            __syncthreads();
            if (threadIdx.x == 0) c.nsnap = k + 1;
            __syncthreads();
        };
        snapshot(0.f);
        for (;;) {
            if (threadIdx.x == 0) {
                bool go = (s_inst.max_steps < 0 || c.n < s_inst.max_steps) && c.simTime < s_inst.max_time;
                if (go) {
                    float mindt = s_next[0];
                    int minspec = 0;
                    for (int i = 1; i < S; ++i)
                        if (s_next[i] < mindt) { mindt = s_next[i]; minspec = i; }
                    int ev = 0;
                    const float mo = c.outputLast + s_inst.output_interval;
                    if (mo < mindt) { mindt = mo; ev = 1; }
                    c.mindt = mindt;
                    c.minspec = minspec;
                    c.ev = ev;
                    c.window = mindt - c.simTime;
                }
                c.stop = go ? 0 : 1;
            }
            __syncthreads();
            if (c.stop) break;
            uint32_t sd = (uint32_t)c.n * 64u;
            if (R > 0) {
                int* x = xs + threadIdx.x;
                int err = 0;
                for (int cell = threadIdx.x; cell < area; cell += NT) {
                    for (int s = 0; s < S; ++s) x[s * NT] = st[(int64_t)s * area + cell];
                    Stream rs;
                    rs.init(key0, key1, sd, (uint32_t)cell, PH_SSA);
                    err |= R > 6 ? ssa_cell_inc(rt, deps, R, x, NT, hs + threadIdx.x, rs, c.window)
                                 : ssa_cell(rt, R, x, NT, rs, c.window);
                    for (int s = 0; s < S; ++s) st[(int64_t)s * area + cell] = x[s * NT];
                }
                if (err) atomicOr(&A.status[id], err);
                sd++;
            }
            __syncthreads();
            if (c.ev == 0) {
                for (int i = 0; i < S; ++i) {
                    if (!(i == c.minspec || s_next[i] <= c.mindt)) continue;
                    if (!(s_next[i] > 0)) continue;
                    int32_t* plane = st + (int64_t)i * area;
                    for (int cell = threadIdx.x; cell < area; cell += NT) {
                        Stream rs;
                        rs.init(key0, key1, sd, (uint32_t)cell, PH_DIFF | ((uint32_t)i << 8));
                        int l[4];
                        homog_lost(plane[cell], pmove, rs, cell % W, cell / W, W, W, bm, l);
                        reinterpret_cast<int4*>(lost)[cell] = make_int4(l[0], l[1], l[2], l[3]);
                    }
                    __syncthreads();
                    for (int cell = threadIdx.x; cell < area; cell += NT) {
                        const int x = cell % W, y = cell / W;
                        const int4 o = reinterpret_cast<const int4*>(lost)[cell];
                        int v = plane[cell] - (o.x + o.y + o.z + o.w);
                        if (x > 0) v += lost[4 * (cell - 1) + 1];
                        if (x < W - 1) v += lost[4 * (cell + 1) + 0];
                        if (y > 0) v += lost[4 * (cell - W) + 3];
                        if (y < W - 1) v += lost[4 * (cell + W) + 2];
                        plane[cell] = v;
                    }
                    __syncthreads();
                    if (threadIdx.x == 0) s_next[i] += s_dt[i];
                }
            } else if (c.simTime >= c.outputLast + s_inst.output_interval) {
                snapshot(c.mindt);
                if (threadIdx.x == 0) c.outputLast += s_inst.output_interval;
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                c.simTime = c.mindt;
                c.n += 1;
                if ((s_inst.flags & GPGMP_FLAG_STOP_ON_ERROR) && *((volatile int32_t*)&A.status[id]) != 0) c.stop = 2;
            }
            __syncthreads();
            if (c.stop == 2) break;
        }
        snapshot(c.simTime);
        if (threadIdx.x == 0) A.steps[id] = c.n;
        __syncthreads();
    }
}

// Poisson(lambda) initial counts per instance, species and cell (same stream as
// the solver's gpgmp_init_poisson for the instance's key)
__global__ void k_ensemble_init(const gpgmp_instance* inst, int n_inst, const float* lambda, int32_t* state) {
    const int id = blockIdx.x;
    if (id >= n_inst) return;
    const gpgmp_instance I = inst[id];
    const int area = I.width * I.width;
    for (int cell = threadIdx.x; cell < area; cell += blockDim.x) {
        for (int s = 0; s < I.num_species; ++s) {
            Stream st;
            st.init(I.seed, I.realisation, 0u, (uint32_t)cell, PH_INIT | ((uint32_t)s << 8));
            state[I.state_offset + (int64_t)s * area + cell] = poisson(st, lambda[I.species_offset + s]);
        }
    }
}

}  // namespace

struct gpgmp_ensemble {
    int n = 0;
    int max_species = 0, max_area = 0, max_reactions = 0;
    std::vector<gpgmp_instance> inst;
    gpgmp_instance* d_inst = nullptr;
    int32_t* d_order = nullptr;
    float* d_diff = nullptr;
    float* d_lambda = nullptr;
    gpgmp_reaction* d_reac = nullptr;
    int32_t* d_status = nullptr;
    int64_t* d_steps = nullptr;
    int64_t* d_snap_time_off = nullptr;
    float* d_snap_times = nullptr;
    int64_t snap_time_total = 0;
    int32_t* d_lost = nullptr;
    unsigned int* d_queue = nullptr;
    int threads = 256, ctas_per_sm = 4, num_sms = 148, grid = 0;
    size_t smem = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int32_t* graph_state = nullptr;
    int32_t* graph_snaps = nullptr;
    cudaStream_t graph_stream = nullptr;
};

#define CK(expr)                                                                                              \
    do {                                                                                                      \
        cudaError_t e_ = (expr);                                                                              \
        if (e_ != cudaSuccess) return set_error(GPGMP_ERR_CUDA, "%s: %s", #expr, cudaGetErrorString(e_));    \
    } while (0)

namespace {

void ens_free(gpgmp_ensemble* h) {
    if (h->exec) cudaGraphExecDestroy(h->exec);
    if (h->graph) cudaGraphDestroy(h->graph);
    void* ptrs[] = {h->d_inst, h->d_order, h->d_diff, h->d_lambda, h->d_reac, h->d_status, h->d_steps,
                    h->d_snap_time_off, h->d_snap_times, h->d_lost, h->d_queue};
    for (void* p : ptrs)
        if (p) cudaFree(p);
}

// longest-processing-time order: cells x species x steps x (1 + reactions / 4)
double est_cost(const gpgmp_instance& I, const float* diffusion) {
    float dmax = 0.f;
    for (int s = 0; s < I.num_species; ++s) dmax = std::max(dmax, diffusion[I.species_offset + s]);
    const double h = (double)I.physical_length / I.width;
    const double dtmin = dmax > 0 ? I.p0 / 6.0 * h * h / dmax : I.max_time;
    const double steps = I.max_time / std::max(dtmin, 1e-9) + 1.0;
    return (double)I.width * I.width * I.num_species * steps * (1.0 + I.num_reactions / 4.0);
}

int configure(gpgmp_ensemble* h, int threads, int ctas_per_sm) {
    if (threads != 128 && threads != 256 && threads != 512 && threads != 1024)
        return set_error(GPGMP_ERR_INVALID, "threads per CTA must be 128, 256, 512 or 1024");
    h->threads = threads;
    h->smem = sizeof(gpgmp_reaction) * MAX_REACTIONS + sizeof(uint32_t) * 4 * MAX_REACTIONS +
              sizeof(int) * (size_t)h->max_species * threads + sizeof(float) * (size_t)h->max_reactions * threads;
    CK(cudaFuncSetAttribute(k_ensemble, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)h->smem));
    int dev = 0, sms = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    int occ = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_ensemble, threads, h->smem));
    if (occ < 1) return set_error(GPGMP_ERR_UNSUPPORTED, "ensemble kernel does not fit an SM");
    h->num_sms = sms;
    h->ctas_per_sm = std::max(1, std::min(ctas_per_sm, occ));
    h->grid = sms * h->ctas_per_sm;
    // lost-count scratch: one slot per CTA
    if (h->d_lost) cudaFree(h->d_lost);
    h->d_lost = nullptr;
    CK(cudaMalloc(&h->d_lost, sizeof(int32_t) * 4 * (size_t)h->max_area * h->grid));
    if (h->exec) { cudaGraphExecDestroy(h->exec); h->exec = nullptr; }
    if (h->graph) { cudaGraphDestroy(h->graph); h->graph = nullptr; }
    return GPGMP_OK;
}

}  // namespace

extern "C" {

int gpgmp_ensemble_create(const gpgmp_instance* instances, int32_t n, const float* diffusion, int64_t n_diffusion,
                          const float* lambda, const gpgmp_reaction* reactions, int64_t n_reactions,
                          gpgmp_ensemble** out) {
    if (!out || !instances || n <= 0 || !diffusion || n_diffusion <= 0 || (n_reactions > 0 && !reactions))
        return set_error(GPGMP_ERR_INVALID, "bad argument");
    *out = nullptr;
    auto* h = new gpgmp_ensemble();
    h->n = n;
    h->inst.assign(instances, instances + n);
    int64_t snap_total = 0;
    std::vector<int64_t> snap_off(n, -1);
    for (int i = 0; i < n; ++i) {
        const gpgmp_instance& I = instances[i];
        if (I.width <= 0 || I.width > 4096 || I.num_species <= 0 || I.num_species > MAX_SPECIES ||
            I.num_reactions < 0 || I.num_reactions > MAX_REACTIONS || I.species_offset < 0 ||
            I.species_offset + I.num_species > n_diffusion || I.reaction_offset < 0 ||
            I.reaction_offset + I.num_reactions > n_reactions || I.state_offset < 0) {
            delete h;
            return set_error(GPGMP_ERR_INVALID, "instance %d is malformed", i);
        }
        for (int r = 0; r < I.num_reactions; ++r) {
            const gpgmp_reaction& rc = reactions[I.reaction_offset + r];
            bool ok = rc.num_reactants >= 0 && rc.num_reactants <= 3 && rc.num_products >= 0 && rc.num_products <= 4;
            for (int j = 0; ok && j < rc.num_reactants; ++j)
                ok = rc.reactant_species[j] >= 0 && rc.reactant_species[j] < I.num_species;
            for (int j = 0; ok && j < rc.num_products; ++j)
                ok = rc.product_species[j] >= 0 && rc.product_species[j] < I.num_species;
            if (!ok) {
                delete h;
                return set_error(GPGMP_ERR_INVALID, "instance %d reaction %d is malformed", i, r);
            }
        }
        h->max_species = std::max(h->max_species, I.num_species);
        h->max_reactions = std::max(h->max_reactions, I.num_reactions);
        h->max_area = std::max(h->max_area, I.width * I.width);
        if (I.snapshot_offset >= 0 && I.max_snapshots > 0) {
            snap_off[i] = snap_total;
            snap_total += I.max_snapshots;
        }
    }
    std::vector<int32_t> order(n);
    for (int i = 0; i < n; ++i) order[i] = i;
    std::vector<double> cost(n);
    for (int i = 0; i < n; ++i) cost[i] = est_cost(instances[i], diffusion);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost[a] > cost[b]; });
    cudaError_t e = cudaSuccess;
    auto A = [&](void** p, size_t b) { if (e == cudaSuccess) e = cudaMalloc(p, b > 0 ? b : 1); };
    A((void**)&h->d_inst, sizeof(gpgmp_instance) * n);
    A((void**)&h->d_order, sizeof(int32_t) * n);
    A((void**)&h->d_diff, sizeof(float) * n_diffusion);
    A((void**)&h->d_lambda, sizeof(float) * n_diffusion);
    A((void**)&h->d_reac, sizeof(gpgmp_reaction) * (n_reactions > 0 ? n_reactions : 1));
    A((void**)&h->d_status, sizeof(int32_t) * n);
    A((void**)&h->d_steps, sizeof(int64_t) * n);
    A((void**)&h->d_snap_time_off, sizeof(int64_t) * n);
    A((void**)&h->d_snap_times, sizeof(float) * (snap_total > 0 ? snap_total : 1));
    A((void**)&h->d_queue, sizeof(unsigned int));
    if (e == cudaSuccess) e = cudaMemcpy(h->d_inst, instances, sizeof(gpgmp_instance) * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(h->d_order, order.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(h->d_diff, diffusion, sizeof(float) * n_diffusion, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && lambda)
        e = cudaMemcpy(h->d_lambda, lambda, sizeof(float) * n_diffusion, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && n_reactions > 0)
        e = cudaMemcpy(h->d_reac, reactions, sizeof(gpgmp_reaction) * n_reactions, cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(h->d_snap_time_off, snap_off.data(), sizeof(int64_t) * n, cudaMemcpyHostToDevice);
    h->snap_time_total = snap_total;
    if (e != cudaSuccess) {
        int c = set_error(e == cudaErrorMemoryAllocation ? GPGMP_ERR_NOMEM : GPGMP_ERR_CUDA, "%s",
                          cudaGetErrorString(e));
        ens_free(h);
        delete h;
        return c;
    }
    int rc = configure(h, 256, 4);
    if (rc) {
        ens_free(h);
        delete h;
        return rc;
    }
    *out = h;
    return GPGMP_OK;
}

int gpgmp_ensemble_destroy(gpgmp_ensemble* h) {
    if (!h) return GPGMP_OK;
    cudaDeviceSynchronize();
    ens_free(h);
    delete h;
    return GPGMP_OK;
}

int gpgmp_ensemble_configure(gpgmp_ensemble* h, int32_t threads_per_cta, int32_t ctas_per_sm) {
    if (!h) return set_error(GPGMP_ERR_INVALID, "handle is NULL");
    return configure(h, threads_per_cta, ctas_per_sm);
}

int gpgmp_ensemble_init_poisson(gpgmp_ensemble* h, int32_t* state, void* stream) {
    if (!h || !state) return set_error(GPGMP_ERR_INVALID, "bad argument");
    k_ensemble_init<<<h->n, 256, 0, (cudaStream_t)stream>>>(h->d_inst, h->n, h->d_lambda, state);
    CK(cudaGetLastError());
    return GPGMP_OK;
}

// Runs every instance to its end time.  The first run with a given (state,
// snapshots, stream) captures the launch into a CUDA graph; later runs replay it.
int gpgmp_ensemble_run(gpgmp_ensemble* h, int32_t* state, int32_t* snapshots, void* stream) {
    if (!h || !state) return set_error(GPGMP_ERR_INVALID, "bad argument");
    cudaStream_t st = (cudaStream_t)stream;
    if (!h->exec || h->graph_state != state || h->graph_snaps != snapshots || h->graph_stream != st) {
        if (h->exec) { cudaGraphExecDestroy(h->exec); h->exec = nullptr; }
        if (h->graph) { cudaGraphDestroy(h->graph); h->graph = nullptr; }
        cudaStream_t cap = nullptr;
        CK(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
        EnsArgs a{};
        a.inst = h->d_inst; a.order = h->d_order; a.diffusion = h->d_diff; a.reactions = h->d_reac;
        a.state = state; a.snapshots = snapshots; a.snap_times = h->d_snap_times;
        a.snap_time_off = h->d_snap_time_off; a.status = h->d_status; a.steps = h->d_steps;
        a.lost = h->d_lost; a.lost_stride = 4 * (int64_t)h->max_area; a.queue = h->d_queue; a.n_inst = h->n;
        a.max_species = h->max_species;
        a.max_reactions = h->max_reactions;
        cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            cudaMemsetAsync(h->d_queue, 0, sizeof(unsigned int), cap);
            cudaMemsetAsync(h->d_status, 0, sizeof(int32_t) * h->n, cap);
            k_ensemble<<<h->grid, h->threads, h->smem, cap>>>(a);
            e = cudaStreamEndCapture(cap, &h->graph);
        }
        cudaStreamDestroy(cap);
        if (e != cudaSuccess) return set_error(GPGMP_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
        CK(cudaGraphInstantiate(&h->exec, h->graph, 0));
        h->graph_state = state;
        h->graph_snaps = snapshots;
        h->graph_stream = st;
    }
    CK(cudaGraphLaunch(h->exec, st));
    return GPGMP_OK;
}

int gpgmp_ensemble_results(gpgmp_ensemble* h, int32_t* status, int64_t* steps, float* snapshot_times) {
    if (!h) return set_error(GPGMP_ERR_INVALID, "handle is NULL");
    CK(cudaDeviceSynchronize());
    if (status) CK(cudaMemcpy(status, h->d_status, sizeof(int32_t) * h->n, cudaMemcpyDeviceToHost));
    if (steps) CK(cudaMemcpy(steps, h->d_steps, sizeof(int64_t) * h->n, cudaMemcpyDeviceToHost));
    if (snapshot_times && h->snap_time_total > 0)
        CK(cudaMemcpy(snapshot_times, h->d_snap_times, sizeof(float) * h->snap_time_total, cudaMemcpyDeviceToHost));
    return GPGMP_OK;
}

int gpgmp_ensemble_launch_shape(gpgmp_ensemble* h, int32_t* threads, int32_t* ctas_per_sm, int32_t* grid) {
    if (!h) return set_error(GPGMP_ERR_INVALID, "handle is NULL");
    if (threads) *threads = h->threads;
    if (ctas_per_sm) *ctas_per_sm = h->ctas_per_sm;
    if (grid) *grid = h->grid;
    return GPGMP_OK;
}

}  // extern "C"
