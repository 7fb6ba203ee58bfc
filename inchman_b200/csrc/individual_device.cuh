// Individual species: molecules tracked one by one (IndividualSolver.cpp,
// IndividualSolver.cl).  Shared by the prebuilt kernels (individual.cu) and by the
// kernels compiled at run time with a model's drift/diffusivity and new-individuals
// methods (jit.cpp), so both run the same code around the model's statements.
//
// An individual species of R realisations is one list of (key, id) pairs sorted by
// key = r * area + cell, with four properties per id (DiffusivityX, DiffusivityY,
// DriftX, DriftY, stored [4][capacity]).  Per individual, as the reference's kernels:
//   sweep   (individual_diffuseX/Y, IndividualSolver.cl:750-1015): the method sees the
//           individual (State = its cell's count of the species, its properties) and
//           the other species as zero dummies; D and r of the sweep direction give the
//           jump probabilities of the inhomogeneous sweep (sweep_probs); one uniform
//           draw per individual moves it one cell or keeps it.  A move across a
//           reflecting wall is cancelled; across an absorbing wall the individual
//           leaves (key = the killed key, its id goes back to the pool).
//   fields  (computeDiffusionConstants, IndividualSolver.cl:654-748): per cell, the
//           largest diffusivity and drift magnitude the method gives its individuals
//           (for the next time step) and the cell's new count.  The sweep folds them in
//           as it moves each individual (atomic maxima and counts), so the list needs no
//           sort per sweep -- it is sorted when the bookkeeping or a reader needs the
//           cell order; the draws are keyed by id, so the results do not depend on it.
//   newborn (updateNewParticles, IndividualSolver.cl:1135-1293): the new-individuals
//           method sets the properties of each individual created by a reaction
//           window; RANDOM is a uniform draw.
// Draws are Philox streams keyed by (seed, realisation) and counted by (step seed,
// id, phase | species << 8 | direction), so they replay on the CPU.
#pragma once
#include "stoch_device.cuh"

namespace gpgmp {

constexpr uint32_t PH_INDIV = 0x08000000u;    // individual sweeps
constexpr uint32_t PH_NEWIND = 0x09000000u;   // properties of new individuals
constexpr int kIndMaxSpecies = 32;

// the reference's _species_t (IndividualSolver.cl:690-697)
struct IndSpecies {
    int State;
    const int* SpeciesState;
    float MeanX;
    float DiffusivityX, DiffusivityY, DriftX, DriftY;
};

struct IndArgs {
    int W, H, S, R, species, dir;
    float L, dx, dt, sim_time;
    int bmask[4];                  // x-, x+, y-, y+ : 0 reflecting, 1 absorbing
    uint32_t seed, step_seed;
    uint32_t* keys;                // list keys (r * area + cell), updated by the sweep
    const uint32_t* ids;
    long long n;
    uint32_t killed_key;           // R * area
    float* props;                  // [4][cap] by id
    long long cap;
    int* planes[kIndMaxSpecies];   // current state buffer of each species ([R][S][area] layout)
    const uint32_t* start;         // per key: first list position (fields)
    const uint32_t* count;         // per key: number of individuals (fields)
    float* fDx;                    // per key: largest DiffusivityX ... (fields)
    float* fDy;
    float* fRx;                    // largest |DriftX|
    float* fRy;
    uint8_t* newborn;              // [cap] flag by id (newborn)
    uint32_t* killed;              // individuals that left in this sweep (sweep)
};

// Where an individual is, for the methods (the same names the field kernels give them).
struct IndPos {
    int GridX, GridY;
    float PhysicalX, PhysicalY, PhysicalSimTime;
};

__device__ __forceinline__ IndPos ind_pos(const IndArgs& a, int cell) {
    IndPos p;
    p.GridX = cell % a.W;
    p.GridY = cell / a.W;
    p.PhysicalX = a.L / (float)a.W * ((float)p.GridX - (float)a.W * 0.5f);
    p.PhysicalY = a.L / (float)a.H * ((float)p.GridY - (float)a.H * 0.5f);
    p.PhysicalSimTime = a.sim_time;
    return p;
}

__device__ __forceinline__ IndSpecies ind_load(const IndArgs& a, uint32_t id, int r, int cell) {
    const long long area = (long long)a.W * a.H;
    IndSpecies sp;
    const int* plane = a.planes[a.species] + ((long long)r * a.S + a.species) * area;
    sp.State = plane[cell];
    sp.SpeciesState = plane;
    sp.MeanX = 0.f;
    sp.DiffusivityX = a.props[id];
    sp.DiffusivityY = a.props[a.cap + id];
    sp.DriftX = a.props[2 * a.cap + id];
    sp.DriftY = a.props[3 * a.cap + id];
    return sp;
}

// The properties as stored (a model without a drift/diffusivity method).
struct IndDriftStored {
    __device__ __forceinline__ void operator()(IndSpecies&, const IndArgs&, const IndPos&) const {}
};
// No new-individuals method: a new individual keeps the properties its id has.
struct IndNewbornKeep {
    static constexpr bool kActive = false;
    __device__ __forceinline__ void operator()(IndSpecies&, const IndArgs&, const IndPos&, Stream&) const {}
};

// largest non-negative float by its bits (they order as unsigned integers)
__device__ __forceinline__ void ind_max_field(float* f, float v) {
    if (v > 0.f) atomicMax(reinterpret_cast<unsigned int*>(f), __float_as_uint(v));
}

template <class DRIFT>
__device__ __forceinline__ void ind_sweep_body(const IndArgs& a, const DRIFT& drift) {
    const long long area = (long long)a.W * a.H;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < a.n;
         i += (long long)gridDim.x * blockDim.x) {
        const uint32_t key = a.keys[i];
        if (key >= a.killed_key) continue;
        const int r = (int)(key / area);
        const int cell = (int)(key - (long long)r * area);
        const uint32_t id = a.ids[i];
        IndSpecies sp = ind_load(a, id, r, cell);
        const IndPos pos = ind_pos(a, cell);
        drift(sp, a, pos);
        const float D = a.dir == 0 ? sp.DiffusivityX : sp.DiffusivityY;
        const float v = a.dir == 0 ? sp.DriftX : sp.DriftY;
        float Pp, Pm;
        sweep_probs(D, v, a.dt, a.dx, &Pp, &Pm);
        Stream st;
        st.init(a.seed, (uint32_t)r, a.step_seed, id, PH_INDIV | ((uint32_t)a.species << 8) | (uint32_t)a.dir);
        const float u = u01(st.next());
        const int mv = u < Pp ? 1 : (u < Pp + Pm ? -1 : 0);
        uint32_t out = key;
        if (mv != 0) {
            const int c = a.dir == 0 ? pos.GridX : pos.GridY;
            const int lim = a.dir == 0 ? a.W : a.H;
            const int nc = c + mv;
            if (nc < 0 || nc >= lim) {
                const int wall = (a.dir == 0 ? 0 : 2) + (mv > 0 ? 1 : 0);
                if (a.bmask[wall] != 0) out = a.killed_key;   // absorbing: the individual leaves
                // reflecting: the move is cancelled
            } else {
                const int ncell = a.dir == 0 ? pos.GridY * a.W + nc : nc * a.W + pos.GridX;
                out = (uint32_t)((long long)r * area + ncell);
            }
            a.keys[i] = out;
        }
        if (out >= a.killed_key) {
            atomicAdd(a.killed, 1u);
            continue;
        }
        // the cell it is in now: its count, and its method's values for the cell's
        // largest diffusivity and drift (computeDiffusionConstants; State is the cell's
        // count before this sweep, as the reference's state buffer still holds it)
        if (a.fDx) {
            const int ncell = (int)(out - (long long)r * area);
            IndSpecies sp2 = ind_load(a, id, r, ncell);
            drift(sp2, a, ind_pos(a, ncell));
            ind_max_field(a.fDx + out, sp2.DiffusivityX);
            ind_max_field(a.fDy + out, sp2.DiffusivityY);
            ind_max_field(a.fRx + out, fabsf(sp2.DriftX));
            ind_max_field(a.fRy + out, fabsf(sp2.DriftY));
            atomicAdd(const_cast<uint32_t*>(a.count) + out, 1u);
        }
    }
}

template <class DRIFT>
__device__ __forceinline__ void ind_fields_body(const IndArgs& a, const DRIFT& drift) {
    const long long area = (long long)a.W * a.H;
    const long long total = (long long)a.R * area;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < total;
         k += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(k / area);
        const int cell = (int)(k - (long long)r * area);
        const uint32_t s0 = a.start[k], cnt = a.count[k];
        float dxm = 0.f, dym = 0.f, rxm = 0.f, rym = 0.f;
        const IndPos pos = ind_pos(a, cell);
        for (uint32_t j = 0; j < cnt; ++j) {
            IndSpecies sp = ind_load(a, a.ids[s0 + j], r, cell);    // State: the count before the sweep
            drift(sp, a, pos);
            dxm = fmaxf(dxm, sp.DiffusivityX);
            dym = fmaxf(dym, sp.DiffusivityY);
            rxm = fmaxf(rxm, fabsf(sp.DriftX));
            rym = fmaxf(rym, fabsf(sp.DriftY));
        }
        a.fDx[k] = dxm;
        a.fDy[k] = dym;
        a.fRx[k] = rxm;
        a.fRy[k] = rym;
    }
}

// the cells' new counts, then the smallest time step of the sweep's direction over
// every cell from the fields the sweep folded in (k_timestep's rule): the key of the
// smallest step goes into *inv_min_key inverted, as an atomic maximum, so that the
// word starts from zero with the others the sweep clears
__device__ __forceinline__ void ind_counts_timestep_body(const IndArgs& a, float dx, int kind, float stay,
                                                         uint32_t* inv_min_key) {
    const long long area = (long long)a.W * a.H;
    const long long total = (long long)a.R * area;
    const float* D = a.dir == 0 ? a.fDx : a.fDy;
    const float* r = a.dir == 0 ? a.fRx : a.fRy;
    uint32_t best = 0u;   // inverted key: larger is a smaller step
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < total;
         k += (long long)gridDim.x * blockDim.x) {
        const int rr = (int)(k / area);
        const long long cell = k - (long long)rr * area;
        a.planes[a.species][((long long)rr * a.S + a.species) * area + cell] = (int)a.count[k];
        const float ts = kind == kTsFpe             ? fpe_timestep(D[k], r[k], dx, stay)
                         : kind == kTsDeterministic ? det_timestep(D[k], r[k], dx)
                                                    : cell_timestep(D[k], r[k], dx);
        if (ts == ts) {   // NaN is skipped, as fminf does
            const uint32_t b = __float_as_uint(ts);
            const uint32_t key = (b & 0x80000000u) ? ~b : (b | 0x80000000u);
            best = ~key > best ? ~key : best;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        const uint32_t other = __shfl_xor_sync(0xffffffffu, best, o);
        best = other > best ? other : best;
    }
    if ((threadIdx.x & 31) == 0 && best) atomicMax(inv_min_key, best);
}

// the cells' new counts, once every thread of the fields pass has read the old ones
__device__ __forceinline__ void ind_counts_body(const IndArgs& a) {
    const long long area = (long long)a.W * a.H;
    const long long total = (long long)a.R * area;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < total;
         k += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(k / area);
        const long long cell = k - (long long)r * area;
        a.planes[a.species][((long long)r * a.S + a.species) * area + cell] = (int)a.count[k];
    }
}

template <class NEWBORN>
__device__ __forceinline__ void ind_newborn_body(const IndArgs& a, const NEWBORN& method) {
    const long long area = (long long)a.W * a.H;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < a.n;
         i += (long long)gridDim.x * blockDim.x) {
        const uint32_t id = a.ids[i];
        if (!a.newborn[id]) continue;
        a.newborn[id] = 0;
        const uint32_t key = a.keys[i];
        const int r = (int)(key / area);
        const int cell = (int)(key - (long long)r * area);
        IndSpecies sp = ind_load(a, id, r, cell);
        Stream st;
        st.init(a.seed, (uint32_t)r, a.step_seed, id, PH_NEWIND | ((uint32_t)a.species << 8));
        method(sp, a, ind_pos(a, cell), st);
        a.props[id] = sp.DiffusivityX;
        a.props[a.cap + id] = sp.DiffusivityY;
        a.props[2 * a.cap + id] = sp.DriftX;
        a.props[3 * a.cap + id] = sp.DriftY;
    }
}

}  // namespace gpgmp
