// Host side of the individual species (individual.cu): the list of one species and
// the steps the solver takes with it.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "individual_device.cuh"
#include "jit.h"

namespace gpgmp {

// One individual species over all realisations: (key, id) pairs sorted by key =
// r * area + cell, double-buffered; the free ids; four properties per id.
struct IndList {
    int species = -1;
    long long cap = 0, ncells = 0;    // capacity in individuals, R * area
    long long n = 0, npool = 0;
    uint32_t* keys[2] = {nullptr, nullptr};
    uint32_t* ids[2] = {nullptr, nullptr};
    uint32_t* pool[2] = {nullptr, nullptr};
    int cur = 0, pcur = 0;
    float* props = nullptr;           // [4][cap]: DiffusivityX, DiffusivityY, DriftX, DriftY
    uint8_t* newborn = nullptr;       // [cap]
    uint32_t* start[2] = {nullptr, nullptr};   // [ncells + 1] first list position per key (+ the killed bin)
    uint32_t* count = nullptr;        // [ncells + 1]
    int32_t* goal = nullptr;          // [ncells + 1] counts to maintain
    float* fields = nullptr;          // [4][ncells]
    uint32_t* d_small = nullptr;      // [2]: individuals that left in the last sweep, its time step key
    void* sweep_block = nullptr;      // one allocation: count, fields, d_small (cleared by one memset per sweep)
    uint32_t* h_small = nullptr;      // pinned [2 slots][2]: d_small of the sweeps of one diffuse call
    void* sort_scratch = nullptr;
    size_t sort_bytes = 0;
    void* scan_scratch = nullptr;
    size_t scan_bytes = 0;
    void* pop_scratch = nullptr;
    size_t pop_bytes = 0;
    int key_bits = 0;
    bool sorted = true;               // the list is in key order (and start/count describe it)
    long long pending = 0;            // left through an absorbing wall, still in the list until sorted
};

// The kernels of a model: prebuilt (no model code) or compiled with its drift /
// diffusivity method and its new-individuals method.
struct IndKernels {
    JitFunction sweep = nullptr, fields = nullptr, newborn = nullptr;
    bool newborn_active = false;
};

// may_leave: a wall is absorbing, so individuals can leave (their key is ncells)
int ind_alloc(IndList& l, int species, long long cap, long long ncells, bool may_leave);
void ind_free(IndList& l);

// Builds the list from the counts of the species in the state (ids 0.. in cell
// order, properties 0 for them and (1, 1, 0, 0) for the ids not yet used, as the
// reference's IndividualSolver constructor fills them), then the fields.
int ind_build(IndList& l, IndArgs a, const IndKernels& k, cudaStream_t st);
// One sweep (a.dir) with the counts and fields folded in, then the new time step of
// that direction (the smallest over every cell of every realisation).  Enqueued only:
// the number that left and the time step land in h_small[slot]; once the stream has
// been synchronised, ind_sweep_result books the departures and returns the time step.
int ind_sweep(IndList& l, IndArgs a, const IndKernels& k, float dx, int ts_kind, float stay, int slot,
              cudaStream_t st);
float ind_sweep_result(IndList& l, int slot);
// After a reaction window: the list follows the counts (population bookkeeping);
// the individuals created get the new-individuals method's properties.
int ind_maintain(IndList& l, IndArgs a, const IndKernels& k, cudaStream_t st);
// Fields only (after the properties changed from the host).
int ind_fields(IndList& l, IndArgs a, const IndKernels& k, cudaStream_t st);
// Puts the list in key order (stable) and drops the individuals that left; the
// sweeps leave it unsorted (they fold counts and fields in directly).
int ind_sort(IndList& l, cudaStream_t st);
// individuals in the list that are still in the domain
inline long long ind_count(const IndList& l) { return l.n - l.pending; }

// run-time compiled variants (jit.cpp)
int jit_ind_kernels(const std::string& defines, const std::string& drift_code, const std::string& newborn_code,
                    int num_species, IndKernels* out);
cudaError_t launch_ind_jit(JitFunction fn, const IndArgs& a, long long work, cudaStream_t st);

}  // namespace gpgmp
