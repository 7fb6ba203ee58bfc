/*
 * oracle/orc_ref.c -- TEST INFRASTRUCTURE ONLY (the oracle).
 *
 * Reference-exact restatement of GPGMP's stochastic and deterministic kernels and
 * of its split-step event loop.  Every function follows the reference source line
 * by line; citations are paths inside the reference project.  Arithmetic follows
 * C's promotion rules for the kernels' double literals (the reference compiled
 * for a CPU), which is what oracle/_ref executes and what tests pin against.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "gpgmp_oracle.h"
#include "orc_math.h"

/* ---- small wrappers exported for the tests --------------------------------- */
void orc_threefry2x32_20(const uint32_t ctr[2], const uint32_t key[2], uint32_t out[2]) {
    orc_threefry2x32_20_inl(ctr, key, out);
}
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    orc_philox4x32_10_inl(ctr, key, out);
}
void orc_philox_fill(uint32_t k0, uint32_t k1, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t* out, int n) {
    orc_stream s;
    orc_stream_init(&s, k0, k1, c1, c2, c3);
    for (int i = 0; i < n; ++i) out[i] = orc_stream_next(&s);
}
void orc_logf_many(const float* x, float* y, int n) { for (int i = 0; i < n; ++i) y[i] = orc_logf(x[i]); }
void orc_expf_many(const float* x, float* y, int n) { for (int i = 0; i < n; ++i) y[i] = orc_expf(x[i]); }
void orc_sincos2pi_many(const float* u, float* s, float* c, int n) {
    for (int i = 0; i < n; ++i) orc_sincos2pi(u[i], &s[i], &c[i]);
}
void orc_binomial_many(uint32_t k0, uint32_t k1, const int32_t* n, const float* p, int32_t* out, int count) {
    for (int i = 0; i < count; ++i) {
        orc_stream s;
        orc_stream_init(&s, k0, k1, 0u, (uint32_t)i, ORC_PH_INIT);
        out[i] = orc_binomial(&s, n[i], p[i]);
    }
}
void orc_poisson_many(uint32_t k0, uint32_t k1, const float* lam, int32_t* out, int count) {
    for (int i = 0; i < count; ++i) {
        orc_stream s;
        orc_stream_init(&s, k0, k1, 0u, (uint32_t)i, ORC_PH_INIT);
        out[i] = orc_poisson(&s, lam[i]);
    }
}

/* ---- constants the reference bakes into its generated kernel header --------- */
/* Solver.cpp:509: "StayProbability = " << (1.-p0) << "f" with std::scientific
 * (Solver.cpp:451), i.e. printed with 6 decimals and read back as a float literal. */
static float printed_float(double v) {
    char buf[64];
    snprintf(buf, sizeof buf, "%e", v);
    return strtof(buf, NULL);
}
/* Reaction.cpp:122: the rate is printed with the default stream format (%g) into the
 * kinetic law and compiled as a double literal. */
static double printed_rate(float rate) {
    char buf[64];
    snprintf(buf, sizeof buf, "%g", (double)rate);
    return strtod(buf, NULL);
}
float orc_ref_stay_probability(const orc_model* m) { return printed_float(1. - (double)m->p0); }
/* Solver.cpp:507: PhysicalCellWidth = L / (Real)W, printed the same way. */
float orc_ref_cell_width(const orc_model* m) {
    return printed_float((double)(m->physical_length / (float)m->width));
}

/* Threefry draw as the kernels do it: c.v[0]++ then one call; the two outputs are
 * read as signed ints and mapped by x * 2^-32 + 0.5 (Solver.cpp:467). */
#define M_RAN_INVM32 2.32830643653869628906e-010
typedef struct { uint32_t key[2]; uint32_t ctr[2]; int32_t r[2]; } ref_rng;
static inline void ref_rng_init(ref_rng* g, uint32_t id, int32_t seed) {
    g->key[0] = id;
    g->key[1] = 0xdecafbadu + (uint32_t)seed;
    g->ctr[0] = 0;
    g->ctr[1] = 0xf00dcafeu;
}
static inline void ref_rng_draw(ref_rng* g) {
    uint32_t out[2];
    g->ctr[0]++;
    orc_threefry2x32_20_inl(g->ctr, g->key, out);
    g->r[0] = (int32_t)out[0];
    g->r[1] = (int32_t)out[1];
}

/* StochasticHomogeneousDiffusion.cl:8-103 (diffuse) and :105-124 (updateState). */
/* The reference keys each cell's Threefry stream on the cell alone
 * (StochasticHomogeneousDiffusion.cl:19-20) and diffuse() does not advance the seed,
 * so species diffused in the same event draw the same uniforms (its defect A.1).
 * orc_ref_set_species_streams(1) keys the stream on cell + species * area instead, as
 * the reference's inhomogeneous sweeps do (StochasticInhomogeneousDriftDiffusion.cl:
 * 448-452): the restatement with that one defect corrected. */
static int g_species_streams = 0;
void orc_ref_set_species_streams(int independent) { g_species_streams = independent; }

void orc_ref_homog_diffuse(const orc_model* m, int32_t* state, int species, int32_t seed, int32_t* lost) {
    const int W = m->width, H = m->height;
    const size_t area = (size_t)W * H;
    int32_t* st = state + (size_t)species * area;
    const float Stay = orc_ref_stay_probability(m);
    const float pi = (float)((1. - Stay) / (2. * 3));
    const float p1 = Stay + pi, p2 = p1 + pi, p3 = p2 + pi, p4 = p3 + pi;
    #pragma omp parallel for schedule(static)
    for (int y = 0; y < H; ++y) {
        for (int x = 0; x < W; ++x) {
            const int gid = x + y * W;
            ref_rng g = {{0, 0}, {0, 0}, {0, 0}};
            ref_rng_init(&g, (uint32_t)gid + (g_species_streams ? (uint32_t)(species * area) : 0u), seed);
            int my_state = st[gid];
            size_t mask[4];
            mask[0] = (x == 0) ? (size_t)m->boundary_mask[0] : 1;
            mask[1] = (x == W - 1) ? (size_t)m->boundary_mask[1] : 1;
            mask[2] = (y == 0) ? (size_t)m->boundary_mask[2] : 1;
            mask[3] = (y == H - 1) ? (size_t)m->boundary_mask[3] : 1;
            int l[4] = {0, 0, 0, 0};
            for (int i = 0; i < my_state; ++i) {
                float rnd;
                if (!(i % 2)) { ref_rng_draw(&g); rnd = (float)(g.r[0] * M_RAN_INVM32 + 0.5); }
                else          { rnd = (float)(g.r[1] * M_RAN_INVM32 + 0.5); }
                size_t dir = 3;
                dir -= (rnd <= p3);
                dir -= (rnd <= p2);
                dir -= (rnd <= p1);
                l[dir] += (int)(mask[dir] * (size_t)(rnd > Stay && rnd <= p4));
            }
            for (int d = 0; d < 4; ++d) lost[4 * gid + d] = l[d];
            st[gid] -= (l[0] + l[1] + l[2] + l[3]);
        }
    }
    #pragma omp parallel for schedule(static)
    for (int y = 0; y < H; ++y) {
        for (int x = 0; x < W; ++x) {
            int s = st[x + y * W];
            if (x > 0) s += lost[4 * ((x - 1) + y * W) + 1];
            if (x < W - 1) s += lost[4 * ((x + 1) + y * W) + 0];
            if (y > 0) s += lost[4 * (x + (y - 1) * W) + 3];
            if (y < H - 1) s += lost[4 * (x + (y + 1) * W) + 2];
            st[x + y * W] = s;
        }
    }
}

/* StochasticHomogeneousDiffusion.cl:128-183; launched over W work-items
 * (HomogeneousSolver.cpp:117-120). */
void orc_ref_source_boundary(const orc_model* m, int32_t* state, int species, int32_t seed, int boundary, int source) {
    const int W = m->width, H = m->height;
    int32_t* st = state + (size_t)species * W * H;
    const float Stay = orc_ref_stay_probability(m);
    const float pi = (float)((1. - Stay) / (2. * 3));
    const float p1 = Stay + pi;
    for (int dev = 0; dev < W; ++dev) {
        ref_rng g = {{0, 0}, {0, 0}, {0, 0}};
        ref_rng_init(&g, (uint32_t)dev, seed);
        int gid = 0;
        switch (boundary) {
            case 0: gid = dev * W; break;
            case 1: gid = (W - 1) + dev * W; break;
            case 2: gid = dev; break;
            default: gid = dev + (H - 1) * W; break;
        }
        for (int i = 0; i < source; ++i) {
            float rnd;
            if (!(i % 2)) { ref_rng_draw(&g); rnd = (float)(g.r[0] * M_RAN_INVM32 + 0.5); }
            else          { rnd = (float)(g.r[1] * M_RAN_INVM32 + 0.5); }
            st[gid] += (rnd > Stay && rnd <= p1);
        }
    }
}

/* Gillespie.cl:4-106 with the code Solver.cpp:843-905 generates for mass-action
 * laws (Reaction.cpp:119-138): h_{i+1} = h_0 + rate * A * (A-1) * ... evaluated in
 * double, reaction picked by the cumulative-hazard masks, stoichiometry applied
 * with the mask as factor. */
static inline double ref_kinetic_law(const orc_reaction* r, double lit, const int32_t* x) {
    double v = lit;
    for (int j = 0; j < r->num_reactants; ++j) {
        int32_t a = x[r->reactant_species[j]];
        v = v * a;
        for (int s = 1; s < r->reactant_stoich[j]; ++s) v = v * (a - s);
    }
    return v;
}

void orc_ref_gillespie(const orc_model* m, int32_t* state, int32_t seed, float deltat) {
    const int W = m->width, H = m->height, S = m->num_species, R = m->num_reactions;
    const size_t area = (size_t)W * H;
    if (R <= 0) return;
    double* lit = (double*)malloc(sizeof(double) * R);
    for (int i = 0; i < R; ++i) lit[i] = printed_rate(m->reactions[i].rate);
    #pragma omp parallel for schedule(dynamic, 16)
    for (int64_t gid = 0; gid < (int64_t)area; ++gid) {
        int32_t x[64];
        float h[130];
        uint32_t on[4];
        orc_cell_reactions(m, (size_t)gid, on);
        for (int s = 0; s < S; ++s) x[s] = state[gid + (size_t)s * area];
        ref_rng g = {{0, 0}, {0, 0}, {0, 0}};
        ref_rng_init(&g, (uint32_t)gid, seed);
        float t = 0.f;
        while (t < deltat) {
            h[0] = 0.f;
            for (int i = 0; i < R; ++i) {
                /* a localised reaction's law is multiplied by the cell's mask value, 1 or 0
                 * (Solver.cpp:852-854) */
                const double law = orc_reaction_on(on, i) ? ref_kinetic_law(&m->reactions[i], lit[i], x) : 0.0;
                h[i + 1] = (float)((double)h[0] + law);
                h[0] = h[i + 1];
            }
            if (h[0] == 0) break;
            ref_rng_draw(&g);
            float r1 = (float)(g.r[0] * M_RAN_INVM32 + 0.5);
            float r2 = (float)((g.r[1] * M_RAN_INVM32 + 0.5) * h[0]);
            /* OpenCL's log of a float argument is the float logarithm (the overload
             * for float; Gillespie.cl:72 `log(1.f/_r1) / _h[0]`, all in float) */
            float dt = logf(1.f / r1) / h[0];
            t += dt;
            if (t < deltat) {
                for (int i = 0; i < R; ++i) {
                    int index = (i == 0) ? (r2 < h[1]) : ((r2 >= h[i]) * (r2 < h[i + 1]));
                    const orc_reaction* rc = &m->reactions[i];
                    for (int j = 0; j < rc->num_reactants; ++j)
                        x[rc->reactant_species[j]] = x[rc->reactant_species[j]] - rc->reactant_stoich[j] * index;
                    for (int j = 0; j < rc->num_products; ++j)
                        x[rc->product_species[j]] = x[rc->product_species[j]] + rc->product_stoich[j] * index;
                }
            }
        }
        for (int s = 0; s < S; ++s) state[gid + (size_t)s * area] = x[s];
    }
    free(lit);
}

/* StochasticInhomogeneousDriftDiffusion.cl:426-557 (diffuseX), :559-685 (diffuseY),
 * :687-723 (updateStateX/Y). */
void orc_ref_inhomog_diffuse(const orc_model* m, int32_t* state, int species, int32_t seed, float dt, int sweep_y,
                             const float* Dx, const float* Dy, const float* rxf, const float* ryf, int32_t* lost) {
    const int W = m->width, H = m->height;
    const size_t area = (size_t)W * H;
    const float deltax = orc_ref_cell_width(m);
    const float deltay = printed_float((double)(m->physical_length / (float)m->height));
    #pragma omp parallel for schedule(static)
    for (int y = 0; y < H; ++y) {
        for (int x = 0; x < W; ++x) {
            const size_t gid = (size_t)x + (size_t)y * W + (size_t)species * area;
            ref_rng g = {{0, 0}, {0, 0}, {0, 0}};
            ref_rng_init(&g, (uint32_t)gid, seed);
            int my_state = state[gid];
            size_t mask[4];
            mask[0] = (x == 0) ? (size_t)m->boundary_mask[0] : 1;
            mask[1] = (x == W - 1) ? (size_t)m->boundary_mask[1] : 1;
            mask[2] = (y == 0) ? (size_t)m->boundary_mask[2] : 1;
            mask[3] = (y == H - 1) ? (size_t)m->boundary_mask[3] : 1;
            int l[4] = {0, 0, 0, 0};
            float diffHere = sweep_y ? Dy[gid] : Dx[gid];
            float rx = sweep_y ? ryf[gid] : rxf[gid];
            float dx = sweep_y ? deltay : deltax;
            float ps = (float)(1. - (dt * (2. * diffHere + rx * rx * dt)) / (dx * dx));
            float p1 = (float)((1. - ps) * (1. + (dx * rx) / (2. * diffHere + rx * rx * dt)) / 2.);
            float p2 = (float)(p1 + (1. - ps) * (1. - (dx * rx) / (2. * diffHere + rx * rx * dt)) / 2.);
            for (int i = 0; i < my_state; ++i) {
                float rnd;
                if (!(i % 2)) { ref_rng_draw(&g); rnd = (float)(g.r[0] * M_RAN_INVM32 + 0.5); }
                else          { rnd = (float)(g.r[1] * M_RAN_INVM32 + 0.5); }
                size_t dir = sweep_y ? 2 : 0;
                dir += (rnd <= p1);
                l[dir] += (int)(mask[dir] * (size_t)(rnd <= p2));
            }
            const size_t cell = (size_t)x + (size_t)y * W;
            for (int d = 0; d < 4; ++d) lost[4 * cell + d] = l[d];
            state[gid] -= (l[0] + l[1] + l[2] + l[3]);
        }
    }
    int32_t* st = state + (size_t)species * area;
    #pragma omp parallel for schedule(static)
    for (int y = 0; y < H; ++y) {
        for (int x = 0; x < W; ++x) {
            int s = st[x + y * W];
            if (!sweep_y) {
                if (x > 0) s += lost[4 * ((x - 1) + y * W) + 1];
                if (x < W - 1) s += lost[4 * ((x + 1) + y * W) + 0];
            } else {
                if (y > 0) s += lost[4 * (x + (y - 1) * W) + 3];
                if (y < H - 1) s += lost[4 * (x + (y + 1) * W) + 2];
            }
            st[x + y * W] = s;
        }
    }
}

/* StochasticInhomogeneousDriftDiffusion.cl:88-230 / :232-379 for the
 * stochastic_inhomogeneous solver (the :130-151 branch), then the block and grid
 * minimum (:200-229, :382-423).  Both sweeps use PhysicalCellWidth as deltax. */
float orc_ref_timestep(const orc_model* m, int species, int sweep_y,
                       const float* Dx, const float* Dy, const float* rxf, const float* ryf, float* per_cell) {
    const size_t area = (size_t)m->width * m->height;
    const float deltax = orc_ref_cell_width(m);
    float best = INFINITY;
    for (size_t c = 0; c < area; ++c) {
        size_t idx = c + (size_t)species * area;
        float diffHere = sweep_y ? Dy[idx] : Dx[idx];
        float rx = sweep_y ? ryf[idx] : rxf[idx];
        float timeStep;
        if (rx == 0) {
            timeStep = (float)(deltax * deltax / (2. * diffHere) * (1. - 2. / 3.));
        } else if (diffHere == 0) {
            timeStep = (float)(deltax / fabs(rx));
        } else {
            /* tanh and sinh of the float epsx are the float functions in OpenCL C
             * (overloads), and their products with floats stay float */
            float epsx = (float)(deltax * rx / (2. * diffHere));
            float temp = (float)(1. + (-1. / (tanhf(epsx) * epsx) + 1. / (sinhf(epsx) * sinhf(epsx))));
            if (temp <= 0) temp = (float)(1. / 3.);
            timeStep = deltax / rx * tanhf(epsx) * temp;
        }
        if (per_cell) per_cell[c] = timeStep;
        best = fminf(best, timeStep);
    }
    return best;
}

/* Deterministic.cl:17-65 with mirror neighbours.  The reference updates d_state in
 * place while other work-items read it; in_place=0 gives the race-free (Jacobi)
 * form every parity test uses, in_place=1 the literal sequential sweep. */
void orc_ref_det_diffuse(const orc_model* m, const float* in, float* out, float dt, int in_place) {
    const int W = m->width, H = m->height, S = m->num_species;
    const size_t area = (size_t)W * H;
    const float dxw = orc_ref_cell_width(m);
    const float dx2 = dxw * dxw;
    const float* src = in_place ? out : in;
    if (in_place && out != in) memcpy(out, in, sizeof(float) * area * S);
    for (int y = 0; y < H; ++y) {
        for (int x = 0; x < W; ++x) {
            for (int i = 0; i < S; ++i) {
                const float* s = src + (size_t)i * area;
                float sleft = x > 0 ? s[(x - 1) + y * W] : s[(x + 1) + y * W];
                float sright = x < W - 1 ? s[(x + 1) + y * W] : s[(x - 1) + y * W];
                float stop = y > 0 ? s[x + (y - 1) * W] : s[x + (y + 1) * W];
                float sbottom = y < W - 1 ? s[x + (y + 1) * W] : s[x + (y - 1) * W];
                float shere = s[x + y * W];
                float slaplace = (float)(stop + sbottom + sleft + sright - 4. * shere);
                float diff = m->diffusion[i];
                out[(size_t)i * area + x + y * W] = shere + dt * diff * slaplace / dx2;
            }
        }
    }
}

/* Deterministic.cl:143-238 with the right-hand side Solver.cpp:922-959 generates:
 * d_i = 0. (+|-) |nu|. * rate * A * B ..., laws from Reaction.cpp:145-162. */
static void ref_rhs(const orc_model* m, const double* lit, const uint32_t* on, float* xs, float* deriv, float off,
                    const float* rk) {
    const int S = m->num_species, R = m->num_reactions;
    for (int j = 0; j < S; ++j) { deriv[j] = 0.f; xs[j] += off * rk[j]; }
    for (int i = 0; i < S; ++i) {
        double acc = 0.;
        for (int r = 0; r < R; ++r) {
            if (!orc_reaction_on(on, r)) continue;      /* mask 0 in this cell (Solver.cpp:946-948) */
            const orc_reaction* rc = &m->reactions[r];
            int net = 0;
            for (int j = 0; j < rc->num_products; ++j) if (rc->product_species[j] == i) net += rc->product_stoich[j];
            for (int j = 0; j < rc->num_reactants; ++j) if (rc->reactant_species[j] == i) net -= rc->reactant_stoich[j];
            if (net == 0) continue;
            double term = (double)abs(net) * lit[r];
            for (int j = 0; j < rc->num_reactants; ++j)
                for (int s = 0; s < rc->reactant_stoich[j]; ++s) term = term * xs[rc->reactant_species[j]];
            acc = net > 0 ? acc + term : acc - term;
        }
        deriv[i] = (float)acc;
    }
    for (int j = 0; j < S; ++j) xs[j] -= off * rk[j];
}

void orc_ref_rk4(const orc_model* m, float* state, float deltat) {
    const int S = m->num_species, R = m->num_reactions;
    const size_t area = (size_t)m->width * m->height;
    if (R <= 0) return;
    double* lit = (double*)malloc(sizeof(double) * R);
    for (int i = 0; i < R; ++i) lit[i] = printed_rate(m->reactions[i].rate);
    #pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < (int64_t)area; ++c) {
        float xs[64], k1[64], k2[64], k3[64], k4[64];
        uint32_t on[4];
        orc_cell_reactions(m, (size_t)c, on);
        for (int i = 0; i < S; ++i) { xs[i] = state[c + (size_t)i * area]; k1[i] = 0.f; }
        const int nmax = 20;
        float dtc = deltat / (float)nmax;
        for (int it = 0; it < nmax; ++it) {
            ref_rhs(m, lit, on, xs, k1, 0.f, k1);
            ref_rhs(m, lit, on, xs, k2, (float)(dtc / 2.), k1);
            ref_rhs(m, lit, on, xs, k3, (float)(dtc / 2.), k2);
            ref_rhs(m, lit, on, xs, k4, dtc, k3);
            for (int j = 0; j < S; ++j) {
                xs[j] = (float)(xs[j] + dtc / 6. * (k1[j] + 2. * k2[j] + 2. * k3[j] + k4[j]));
                if (xs[j] < 0.) xs[j] = 0.f;
            }
        }
        for (int i = 0; i < S; ++i) state[c + (size_t)i * area] = xs[i];
    }
    free(lit);
}

/* DiffusionModel.cpp:1414-1603 for stochastic_homogeneous, with HomogeneousSolver's
 * time steps (HomogeneousSolver.cpp:150-166) and diffuse() (:203-235).  The
 * reference seeds step n with boost::uniform_int(mt19937)+n, re-seeded from
 * time(0); this restatement takes a hash of (seed_base, n) instead. */
static inline uint32_t orc_hash32(uint32_t a, uint32_t b) {
    uint32_t h = a * 0x9E3779B1u ^ (b + 0x7F4A7C15u);
    h ^= h >> 16; h *= 0x85EBCA6Bu; h ^= h >> 13; h *= 0xC2B2AE35u; h ^= h >> 16;
    return h;
}

int orc_ref_solve(const orc_model* m, int32_t* state, uint32_t seed_base,
                  int32_t* snaps, float* snap_times, int max_snaps, int* nsnap, int64_t* steps_out) {
    const int S = m->num_species;
    const size_t area = (size_t)m->width * m->height;
    const float h = m->physical_length / (float)m->width;
    float* dtv = (float*)malloc(sizeof(float) * S);
    float* next = (float*)malloc(sizeof(float) * S);
    int32_t* lost = (int32_t*)malloc(sizeof(int32_t) * 4 * area);
    for (int i = 0; i < S; ++i) {
        if (m->diffusion[i] > 0) dtv[i] = m->p0 / ((float)2. * 3) * h * h / m->diffusion[i];
        else dtv[i] = m->max_time;
        next[i] = dtv[i];
    }
    int ns = 0;
#define SNAP(t) do { if (ns < max_snaps) { memcpy(snaps + (size_t)ns * S * area, state, sizeof(int32_t) * S * area); \
                      snap_times[ns] = (t); } ns++; } while (0)
    SNAP(0.f);
    float simTime = 0.f, outputLast = 0.f;
    int64_t n = 0;
    while ((m->max_steps < 0 || n < m->max_steps) && simTime < m->max_time) {
        int32_t seed = (int32_t)(orc_hash32(seed_base, (uint32_t)n) & 0x7fffffffu);
        n++;
        float mindt = next[0];
        int minspec = 0;
        for (int i = 1; i < S; ++i) if (next[i] < mindt) { mindt = next[i]; minspec = i; }
        int ev = 0; /* 0 diffusion, 1 output */
        float mo = outputLast + m->output_interval;
        if (mo < mindt) { mindt = mo; ev = 1; }
        float deltat = mindt - simTime;
        if (m->num_reactions > 0) { orc_ref_gillespie(m, state, seed, deltat); seed++; }
        if (ev == 0) {
            for (int i = 0; i < S; ++i) {
                if (i == minspec || next[i] <= mindt) {
                    if (next[i] > 0) {
                        orc_ref_homog_diffuse(m, state, i, seed, lost);
                        if (m->source_mask[0] > 0) orc_ref_source_boundary(m, state, i, seed, 0, m->source_mask[1]);
                        if (m->source_mask[1] > 0) orc_ref_source_boundary(m, state, i, seed, 1, m->source_mask[1]);
                        if (m->source_mask[2] > 0) orc_ref_source_boundary(m, state, i, seed, 2, m->source_mask[2]);
                        if (m->source_mask[3] > 0) orc_ref_source_boundary(m, state, i, seed, 3, m->source_mask[3]);
                        next[i] += dtv[i];
                    }
                }
            }
        } else {
            if (simTime >= outputLast + m->output_interval) {
                SNAP(mindt);
                outputLast += m->output_interval;
            }
        }
        simTime = mindt;
    }
    SNAP(simTime);
#undef SNAP
    *nsnap = ns;
    *steps_out = n;
    free(dtv); free(next); free(lost);
    return 0;
}

/* DiffusionModel.cpp:1414-1603 for stochastic_inhomogeneous with a linear drift /
 * diffusivity field (Dx, Dy, rx, ry: [S][H][W], the arrays computeDiffusivityDrift
 * fills once): first time steps per species and direction from the per-cell
 * minimum (InhomogeneousSolver.cpp:193-212, StochasticInhomogeneousDriftDiffusion.cl:
 * 124-151 and the block reduction), next diffusion time of a species = the earlier of
 * its x and y clocks (:238-252), diffuse() sweeps x when its clock is due, then y
 * (:254-427), each sweep with the step's seed, which then advances; the time steps
 * stay fixed (no nonlinear method).  Seeds as orc_ref_solve. */
int orc_ref_solve_inhom(const orc_model* m, int32_t* state, uint32_t seed_base, const float* Dx, const float* Dy,
                        const float* rx, const float* ry, int32_t* snaps, float* snap_times, int max_snaps,
                        int* nsnap, int64_t* steps_out) {
    const int S = m->num_species;
    const size_t area = (size_t)m->width * m->height;
    float* dtx = (float*)malloc(sizeof(float) * S);
    float* dty = (float*)malloc(sizeof(float) * S);
    float* nx = (float*)malloc(sizeof(float) * S);
    float* ny = (float*)malloc(sizeof(float) * S);
    int32_t* lost = (int32_t*)malloc(sizeof(int32_t) * 4 * area);
    for (int i = 0; i < S; ++i) {
        dtx[i] = orc_ref_timestep(m, i, 0, Dx, Dy, rx, ry, NULL);
        dty[i] = orc_ref_timestep(m, i, 1, Dx, Dy, rx, ry, NULL);
        nx[i] = dtx[i];
        ny[i] = dty[i];
    }
    int ns = 0;
#define SNAP(t) do { if (ns < max_snaps) { memcpy(snaps + (size_t)ns * S * area, state, sizeof(int32_t) * S * area); \
                      snap_times[ns] = (t); } ns++; } while (0)
    SNAP(0.f);
    float simTime = 0.f, outputLast = 0.f;
    int64_t n = 0;
    while ((m->max_steps < 0 || n < m->max_steps) && simTime < m->max_time) {
        int32_t seed = (int32_t)(orc_hash32(seed_base, (uint32_t)n) & 0x7fffffffu);
        n++;
        float mindt = nx[0] < ny[0] ? nx[0] : ny[0];
        int minspec = 0;
        for (int i = 1; i < S; ++i) {
            const float t = nx[i] < ny[i] ? nx[i] : ny[i];
            if (t < mindt) { mindt = t; minspec = i; }
        }
        int ev = 0;
        const float mo = outputLast + m->output_interval;
        if (mo < mindt) { mindt = mo; ev = 1; }
        const float deltat = mindt - simTime;
        if (m->num_reactions > 0) { orc_ref_gillespie(m, state, seed, deltat); seed++; }
        if (ev == 0) {
            for (int i = 0; i < S; ++i) {
                const float t = nx[i] < ny[i] ? nx[i] : ny[i];
                if (!(i == minspec || t <= mindt) || !(t > 0)) continue;
                if (nx[i] <= mindt) {
                    orc_ref_inhomog_diffuse(m, state, i, seed, dtx[i], 0, Dx, Dy, rx, ry, lost);
                    seed++;
                    nx[i] += dtx[i];
                }
                if (ny[i] <= mindt) {
                    orc_ref_inhomog_diffuse(m, state, i, seed, dty[i], 1, Dx, Dy, rx, ry, lost);
                    seed++;
                    ny[i] += dty[i];
                }
            }
        } else if (simTime >= outputLast + m->output_interval) {
            SNAP(mindt);
            outputLast += m->output_interval;
        }
        simTime = mindt;
    }
    SNAP(simTime);
#undef SNAP
    *nsnap = ns;
    *steps_out = n;
    free(dtx); free(dty); free(nx); free(ny); free(lost);
    return 0;
}

/* R reference-exact runs (homogeneous, or inhomogeneous with fields when Dx is not
 * NULL) from one initial state, OpenMP over the runs (seed base seed_base + 7919 r);
 * every run's first max_snaps snapshots go to snaps [R][max_snaps][S][H][W]. */
void orc_ref_solve_many_snaps(const orc_model* m, const int32_t* init, int R, uint32_t seed_base, const float* Dx,
                              const float* Dy, const float* rx, const float* ry, int max_snaps, int32_t* snaps) {
    const size_t block = (size_t)m->num_species * m->width * m->height;
    #pragma omp parallel for schedule(dynamic, 1)
    for (int r = 0; r < R; ++r) {
        int32_t* st = (int32_t*)malloc(sizeof(int32_t) * block);
        memcpy(st, init, sizeof(int32_t) * block);
        float* t = (float*)malloc(sizeof(float) * (size_t)max_snaps);
        int ns;
        int64_t steps;
        int32_t* out = snaps + (size_t)r * max_snaps * block;
        if (Dx) orc_ref_solve_inhom(m, st, seed_base + (uint32_t)r * 7919u, Dx, Dy, rx, ry, out, t, max_snaps, &ns,
                                    &steps);
        else orc_ref_solve(m, st, seed_base + (uint32_t)r * 7919u, out, t, max_snaps, &ns, &steps);
        free(st);
        free(t);
    }
}

/* R independent reference-exact runs from the same initial state (OpenMP over the
 * runs, seed base seed_base + r); final states only.  For statistical comparisons. */
#include <omp.h>
void orc_ref_solve_many(const orc_model* m, const int32_t* init, int R, uint32_t seed_base, int32_t* finals) {
    const size_t block = (size_t)m->num_species * m->width * m->height;
    #pragma omp parallel for schedule(dynamic, 1)
    for (int r = 0; r < R; ++r) {
        int32_t* st = finals + (size_t)r * block;
        memcpy(st, init, sizeof(int32_t) * block);
        int32_t* snaps = (int32_t*)malloc(sizeof(int32_t) * block);
        float t;
        int ns;
        int64_t steps;
        orc_ref_solve(m, st, seed_base + (uint32_t)r * 7919u, snaps, &t, 1, &ns, &steps);
        free(snaps);
    }
}
