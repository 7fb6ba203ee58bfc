// A compiled C++ consumer of the C ABI (include/gpgmp_c.h), linked against
// libgpgmp_b200.so: it drives the reference's event loop, DiffusionModel::oclSolve
// (exec/src/gpgmp/src/DiffusionModel.cpp:1479-1603), through the Solver members the
// reference calls -- doReactions (gpgmp_do_reactions), getNextDiffusionTime
// (gpgmp_next_diffusion_time) and diffuse (gpgmp_diffuse) -- exactly as a maintainer's
// adapter in place of HomogeneousSolver / InhomogeneousSolver would, and checks that
// its snapshots equal those of gpgmp_solve, the same loop run inside the library.
//
//   oclsolve_loop homogeneous|inhomogeneous
//
// Prints one line and exits 0 when every snapshot, snapshot time and the step count
// agree, 1 when they differ, 2 on an API error.  Step n of the loop uses the seed
// 64 n, the library's schedule (the reference draws uniform_int + n from a Boost
// Mersenne twister seeded by the clock, DiffusionModel.cpp:1467-1482).
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include "gpgmp_c.h"

namespace {

int fail(const char* what, int rc) {
    std::printf("error: %s failed (%d): %s\n", what, rc, gpgmp_last_error());
    return 2;
}

#define CALL(expr)                              \
    do {                                        \
        int rc_ = (expr);                       \
        if (rc_ != GPGMP_OK) return fail(#expr, rc_); \
    } while (0)

gpgmp_reaction reaction(float rate, std::vector<std::pair<int, int>> re, std::vector<std::pair<int, int>> pr) {
    gpgmp_reaction r{};
    r.rate = rate;
    r.num_reactants = (int)re.size();
    for (size_t i = 0; i < re.size(); ++i) { r.reactant_species[i] = re[i].first; r.reactant_stoich[i] = re[i].second; }
    r.num_products = (int)pr.size();
    for (size_t i = 0; i < pr.size(); ++i) { r.product_species[i] = pr[i].first; r.product_stoich[i] = pr[i].second; }
    return r;
}

// The event loop of oclSolve over one solver: next diffusion times, the earliest
// event (diffusion or output, ties to diffusion), the reaction window up to it, the
// due species' diffusion, output snapshots.
int ocl_solve(gpgmp_solver* h, const gpgmp_model_desc& m, size_t block, std::vector<int32_t>& snaps,
              std::vector<float>& times, long long* steps) {
    const int S = m.num_species;
    std::vector<float> dt(S);
    CALL(gpgmp_next_diffusion_time(h, dt.data()));
    std::vector<int32_t> state(block);
    auto snapshot = [&](float t) -> int {
        CALL(gpgmp_get_state(h, state.data()));
        snaps.insert(snaps.end(), state.begin(), state.end());
        times.push_back(t);
        return 0;
    };
    if (int e = snapshot(0.f)) return e;
    float simTime = 0.f, outputLast = 0.f;
    long long n = 0;
    while ((m.max_steps < 0 || n < m.max_steps) && simTime < m.max_time) {
        int seed = (int)((unsigned)n * 64u);
        n++;
        int minspec = 0;
        float mindt = dt[0];
        for (int i = 1; i < S; ++i)
            if (dt[i] < mindt) { mindt = dt[i]; minspec = i; }
        bool output = false;
        const float mindtOutput = outputLast + m.output_interval;
        if (mindtOutput < mindt) { mindt = mindtOutput; output = true; }
        const float deltat = mindt - simTime;
        if (m.num_reactions > 0) CALL(gpgmp_do_reactions(h, deltat, &seed));
        if (!output) {
            for (int i = 0; i < S; ++i)
                if ((i == minspec || dt[i] <= mindt) && dt[i] > 0) CALL(gpgmp_diffuse(h, i, mindt, &seed));
            CALL(gpgmp_next_diffusion_time(h, dt.data()));
        } else if (simTime >= outputLast + m.output_interval) {
            if (int e = snapshot(mindt)) return e;
            outputLast += m.output_interval;
        }
        simTime = mindt;
    }
    if (int e = snapshot(simTime)) return e;
    *steps = n;
    return 0;
}

}  // namespace

int main(int argc, char** argv) {
    const std::string kind = argc > 1 ? argv[1] : "homogeneous";
    const bool inhom = kind == "inhomogeneous";
    // A + B <-> C (config 1's network) on a 20 x 14 grid, one absorbing wall; the
    // inhomogeneous form moves with the built-in Ornstein-Uhlenbeck drift method
    std::vector<float> D = {1.0f, 1.0f, 0.5f};
    std::vector<gpgmp_reaction> rx = {reaction(0.01f, {{0, 1}, {1, 1}}, {{2, 1}}),
                                      reaction(0.1f, {{2, 1}}, {{0, 1}, {1, 1}})};
    gpgmp_model_desc m{};
    m.width = 20; m.height = 14; m.num_species = 3; m.num_reactions = 2;
    m.physical_length = 20.f; m.p0 = 0.1f; m.max_time = 0.6f; m.output_interval = 0.2f; m.max_steps = -1;
    m.boundary_mask[1] = 1;
    m.solver_type = inhom ? GPGMP_STOCHASTIC_INHOMOGENEOUS : GPGMP_STOCHASTIC_HOMOGENEOUS;
    m.drift_method = inhom ? GPGMP_DRIFT_ORNSTEIN_UHLENBECK : GPGMP_DRIFT_HOMOGENEOUS;
    const float ou[8] = {0.8f, 0.6f, 0.3f, 0.1f, 0.05f, 0.2f, 0.f, 0.f};
    std::memcpy(m.drift_params, ou, sizeof ou);
    m.diffusion = D.data();
    m.reactions = rx.data();
    const int R = 2;
    const unsigned seed = 2024;
    const size_t block = (size_t)R * m.num_species * m.width * m.height;

    gpgmp_solver *a = nullptr, *b = nullptr;
    CALL(gpgmp_solver_create(&m, R, seed, 0, &a));
    CALL(gpgmp_solver_create(&m, R, seed, 0, &b));
    const float lambda[3] = {60.f, 40.f, 5.f};
    CALL(gpgmp_init_poisson(a, lambda));
    std::vector<int32_t> init(block);
    CALL(gpgmp_get_state(a, init.data()));
    CALL(gpgmp_set_state(b, init.data()));

    std::vector<int32_t> snaps;
    std::vector<float> times;
    long long steps = 0;
    if (int e = ocl_solve(a, m, block, snaps, times, &steps)) return e;

    const int max_snaps = 16;
    std::vector<int32_t> lib_snaps(block * max_snaps);
    std::vector<float> lib_times(max_snaps);
    int ns = 0;
    long long lib_steps = 0;
    static_assert(sizeof(long long) == sizeof(int64_t), "int64");
    CALL(gpgmp_solve(b, lib_snaps.data(), lib_times.data(), max_snaps, &ns, (int64_t*)&lib_steps));

    bool same = steps == lib_steps && (int)times.size() == ns;
    for (int k = 0; same && k < ns; ++k) {
        same = times[k] == lib_times[k] &&
               std::memcmp(snaps.data() + k * block, lib_snaps.data() + k * block, block * sizeof(int32_t)) == 0;
    }
    long long total = 0;
    for (size_t i = 0; i < block; ++i) total += snaps[snaps.size() - block + i];
    gpgmp_solver_destroy(a);
    gpgmp_solver_destroy(b);
    std::printf("%s: %lld steps, %d snapshots, final total %lld: %s\n", kind.c_str(), steps, (int)times.size(), total,
                same ? "identical to gpgmp_solve" : "DIFFERENT from gpgmp_solve");
    return same ? 0 : 1;
}
