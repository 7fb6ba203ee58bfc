"""CPU checks of the oracle itself: elementary functions against numpy / math,
samplers against their distributions, sort/scan against numpy, the reference's
cell-index semantics, and the replay's statistics against the reference-exact
restatement (same model, different random streams)."""
import math

import numpy as np
import pytest

import oracle
from helpers import small_homog


def test_logf_accuracy():
    x = np.concatenate([np.linspace(1e-7, 1.0, 20001), np.float32(2.0) ** np.arange(-24, 0)]).astype(np.float32)
    y = np.zeros_like(x)
    oracle.orc().orc_logf_many(oracle.ptr(x), oracle.ptr(y), x.size)
    ref = np.log(x.astype(np.float64))
    ulp = np.spacing(np.abs(ref).astype(np.float32)).astype(np.float64)
    assert np.max(np.abs(y - ref) / np.maximum(ulp, 1e-30)) <= 3.0   # within 3 ulp


def test_expf_accuracy():
    x = np.linspace(-80, 80, 40001).astype(np.float32)
    y = np.zeros_like(x)
    oracle.orc().orc_expf_many(oracle.ptr(x), oracle.ptr(y), x.size)
    ref = np.exp(x.astype(np.float64))
    assert np.max(np.abs(y - ref) / ref) < 3e-7


def test_sincos_accuracy():
    u = (np.arange(1 << 16, dtype=np.float64) / (1 << 16)).astype(np.float32)
    s = np.zeros_like(u)
    c = np.zeros_like(u)
    oracle.orc().orc_sincos2pi_many(oracle.ptr(u), oracle.ptr(s), oracle.ptr(c), u.size)
    assert np.max(np.abs(s - np.sin(2 * np.pi * u.astype(np.float64)))) < 3e-7
    assert np.max(np.abs(c - np.cos(2 * np.pi * u.astype(np.float64)))) < 3e-7


@pytest.mark.parametrize("n,p", [(10, 0.3), (100, 0.0667), (1000, 0.5), (50, 0.9), (5000, 0.02), (3, 1.0), (7, 0.0)])
def test_binomial_moments(n, p):
    count = 200_000
    nn = np.full(count, n, np.int32)
    pp = np.full(count, p, np.float32)
    out = np.zeros(count, np.int32)
    oracle.orc().orc_binomial_many(7, 1, oracle.ptr(nn), oracle.ptr(pp), oracle.ptr(out), count)
    assert out.min() >= 0 and out.max() <= n
    mean, var = out.mean(), out.var()
    m0, v0 = n * p, n * p * (1 - p)
    assert abs(mean - m0) <= 5 * math.sqrt(max(v0, 1e-12) / count) + 1e-12
    if v0 > 0:
        assert abs(var / v0 - 1) < 0.03


def test_binomial_pmf_chi2():
    from scipy import stats
    n, p, count = 40, 0.15, 400_000
    out = np.zeros(count, np.int32)
    oracle.orc().orc_binomial_many(3, 9, oracle.ptr(np.full(count, n, np.int32)), oracle.ptr(np.full(count, p, np.float32)),
                                   oracle.ptr(out), count)
    obs = np.bincount(out, minlength=n + 1)
    exp = stats.binom.pmf(np.arange(n + 1), n, p) * count
    keep = exp > 5
    chi2 = ((obs[keep] - exp[keep]) ** 2 / exp[keep]).sum()
    assert stats.chi2.sf(chi2, keep.sum() - 1) > 1e-4


@pytest.mark.parametrize("lam", [0.5, 10.0, 100.0, 200.0])
def test_poisson_moments(lam):
    count = 100_000
    out = np.zeros(count, np.int32)
    oracle.orc().orc_poisson_many(11, 2, oracle.ptr(np.full(count, lam, np.float32)), oracle.ptr(out), count)
    assert abs(out.mean() - lam) < 5 * math.sqrt(lam / count)
    assert abs(out.var() / lam - 1) < 0.03


def test_sort_and_scan_against_numpy():
    rng = np.random.default_rng(0)
    n = 200_000
    keys = rng.integers(0, 5000, size=n).astype(np.uint32)
    vals = np.arange(n, dtype=np.uint32)
    k, v = keys.copy(), vals.copy()
    oracle.orc().orc_sort_pairs_u32(oracle.ptr(k), oracle.ptr(v), n)
    order = np.argsort(keys, kind="stable")
    assert np.array_equal(k, keys[order]) and np.array_equal(v, vals[order])
    x = rng.integers(0, 2**32, size=n, dtype=np.uint64).astype(np.uint32)
    out = np.zeros(n, np.uint32)
    oracle.orc().orc_exclusive_scan_u32(oracle.ptr(x), oracle.ptr(out), n)
    want = (np.concatenate([[0], np.cumsum(x.astype(np.uint64))[:-1]]) % 2**32).astype(np.uint32)
    assert np.array_equal(out, want)


def test_reference_cell_indices_from_offsets():
    """The reference's computeCellIndices ranges equal (start, start + count - 1), with
    empty cells pointing at the next particle."""
    rng = np.random.default_rng(1)
    ncells, n = 300, 1000
    keys = np.sort(rng.integers(5, ncells - 7, size=n).astype(np.uint32))
    keys[100:150] = keys[99]
    left, right = np.zeros(ncells, np.uint32), np.zeros(ncells, np.uint32)
    oracle.orc().orc_cell_indices_ref(oracle.ptr(keys), n, ncells, oracle.ptr(left), oracle.ptr(right))
    start, count = np.zeros(ncells, np.uint32), np.zeros(ncells, np.uint32)
    oracle.orc().orc_cell_offsets(oracle.ptr(keys), n, ncells, oracle.ptr(start), oracle.ptr(count))
    assert np.array_equal(left, start)
    assert np.array_equal(right, np.where(count > 0, start + count - 1, start))


def test_replay_matches_reference_statistics():
    """Homogeneous SSA + diffusion: the replay (binomial jumps, Philox) and the
    reference-exact restatement (one Threefry uniform per particle) have the same
    per-cell mean and variance over realisations (z-tests, Bonferroni over cells
    and species)."""
    from scipy import stats
    m = small_homog(W=6, H=5, max_time=0.3, bmask=(0, 1, 0, 0))
    desc, keep = m.to_desc()
    R = 1200
    lam = [s.initial for s in m.species]
    init = oracle.init_poisson(m.width, m.height, m.num_species, 1, 99, lam)
    rep = np.zeros((R,) + init.shape[1:], np.int64)
    ref = np.zeros_like(rep)
    st, _, _, _, _ = oracle.rep_solve(desc, np.repeat(init, R, axis=0), R, 4321, 1)
    rep[:] = st
    for r in range(R):
        s2, _, _, _ = oracle.ref_solve(desc, init, 1000 + r, 1)
        ref[r] = s2[0]
    a, b = rep.reshape(R, -1).astype(np.float64), ref.reshape(R, -1).astype(np.float64)
    se = np.sqrt(a.var(0, ddof=1) / R + b.var(0, ddof=1) / R) + 1e-12
    z = np.abs(a.mean(0) - b.mean(0)) / se
    alpha = 1e-3 / z.size
    assert (z < stats.norm.isf(alpha / 2)).all(), z.max()
    f = a.var(0, ddof=1) / np.maximum(b.var(0, ddof=1), 1e-12)
    lo, hi = stats.f.ppf(alpha / 2, R - 1, R - 1), stats.f.isf(alpha / 2, R - 1, R - 1)
    ok = (b.var(0) == 0) | ((f > lo) & (f < hi))
    assert ok.all()


def test_localised_replay_matches_reference_statistics():
    """Localised reactions (the reference's reaction mask): the replay and the
    reference-exact restatement agree in per-cell mean and variance, and both leave
    the reactions off outside their regions."""
    from scipy import stats
    from inchman_b200 import _lib
    from inchman_b200.model import DiffusionModel
    m = DiffusionModel(width=6, height=5, physical_length=6.0, p0=0.1, max_time=0.3, output_interval=0.2,
                       solver=_lib.STOCHASTIC_HOMOGENEOUS)
    m.add_species("A", 1.0, 40.0).add_species("B", 1.0, 30.0).add_species("C", 0.5, 5.0)
    m.add_reaction("bind", {"A": 1, "B": 1}, {"C": 1}, 0.02, regions=[(0, 0, 2, 4)])
    m.add_reaction("unbind", {"C": 1}, {"A": 1, "B": 1}, 0.3, regions=[(4, 1, 5, 2)])
    m.add_reaction("src", {}, {"C": 1}, 15.0, regions=[(5, 4, 5, 4)])
    desc, keep = m.to_desc()
    R = 1200
    lam = [s.initial for s in m.species]
    init = oracle.init_poisson(m.width, m.height, m.num_species, 1, 7, lam)
    st, _, _, _, _ = oracle.rep_solve(desc, np.repeat(init, R, axis=0), R, 99, 1)
    rep = st.astype(np.int64)
    ref = np.zeros_like(rep)
    for r in range(R):
        s2, _, _, _ = oracle.ref_solve(desc, init, 5000 + r, 1)
        ref[r] = s2[0]
    a, b = rep.reshape(R, -1).astype(np.float64), ref.reshape(R, -1).astype(np.float64)
    se = np.sqrt(a.var(0, ddof=1) / R + b.var(0, ddof=1) / R) + 1e-12
    z = np.abs(a.mean(0) - b.mean(0)) / se
    alpha = 1e-3 / z.size
    assert (z < stats.norm.isf(alpha / 2)).all(), z.max()
    f = a.var(0, ddof=1) / np.maximum(b.var(0, ddof=1), 1e-12)
    lo, hi = stats.f.ppf(alpha / 2, R - 1, R - 1), stats.f.isf(alpha / 2, R - 1, R - 1)
    assert ((b.var(0) == 0) | ((f > lo) & (f < hi))).all()


def test_localised_reactions_stay_off_outside_their_regions_on_the_cpu():
    """One reaction window: cells outside a reaction's region keep their counts in the
    reference-exact restatement, the replay and the deterministic RK4."""
    from inchman_b200 import _lib
    from inchman_b200.model import DiffusionModel
    W = H = 8
    m = DiffusionModel(width=W, height=H, physical_length=8.0, p0=0.1, max_time=0.5, output_interval=0.5,
                       solver=_lib.STOCHASTIC_HOMOGENEOUS)
    m.add_species("A", 0.0, 30.0).add_species("B", 0.0, 0.0)
    m.add_reaction("conv", {"A": 1}, {"B": 1}, 3.0, regions=[(1, 1, 3, 2)])
    desc, keep = m.to_desc()
    inside = m.reaction_mask()[0].astype(bool)
    init = np.zeros((1, 2, H, W), np.int32)
    init[0, 0] = 30
    st = init.copy()
    oracle.orc().orc_rep_ssa(oracle.model_ptr(desc), oracle.ptr(st), 1, 3, 0, 0.5, None)
    assert (st[0, 0][~inside] == 30).all() and (st[0, 0][inside] < 30).all()
    assert (st[0, 1][~inside] == 0).all() and (st[0].sum(axis=0) == 30).all()
    st = init.copy()
    oracle.orc().orc_ref_gillespie(oracle.model_ptr(desc), oracle.ptr(st), 17, 0.5)
    assert (st[0, 0][~inside] == 30).all() and (st[0, 0][inside] < 30).all()
    m.solver = _lib.DETERMINISTIC_RK4
    desc, keep = m.to_desc()
    fs = np.ascontiguousarray(init[0].astype(np.float32))
    oracle.orc().orc_ref_rk4(oracle.model_ptr(desc), oracle.ptr(fs), 0.5)
    assert (fs[0][~inside] == 30).all() and (fs[0][inside] < 30).all()
    np.testing.assert_allclose(fs.sum(axis=0), 30.0, rtol=1e-6)


def _c3_shaped(W=6, max_time=0.3, seed=3):
    """Lotka-Volterra kinetics, lognormal(0, 0.5) diffusivity and a sinusoidal drift
    kept away from zero (0.25 +- 0.1), reflecting walls: the drift-diffusion model of
    the 512 x 512 workload at test size.  The fields are symmetric under x <-> y (D
    symmetric, rx = f(y), ry = f(x)), so the smallest time steps of the two directions
    are the same number in the reference's float formula and in the solver's double
    one, and both sweep x and y in the same events; with unequal steps the order of
    the two clocks' events depends on the last bits of the time steps."""
    H = W
    from inchman_b200 import _lib
    from inchman_b200.model import DiffusionModel
    m = DiffusionModel(width=W, height=H, physical_length=float(W), p0=0.1, max_time=max_time,
                       output_interval=max_time / 2, solver=_lib.STOCHASTIC_INHOMOGENEOUS,
                       drift_method=_lib.DRIFT_FIELD)
    m.add_species("X", 1.0, 30.0).add_species("Y", 1.0, 30.0)
    m.add_reaction("birth", {"X": 1}, {"X": 2}, 1.0)
    m.add_reaction("predation", {"X": 1, "Y": 1}, {"Y": 2}, 0.005)
    m.add_reaction("death", {"Y": 1}, {}, 0.6)
    rng = np.random.Generator(np.random.PCG64(seed))
    D = rng.lognormal(0.0, 0.5, size=(H, W))
    D = np.triu(D) + np.triu(D, 1).T
    D = D.astype(np.float32)
    y, x = np.meshgrid(np.arange(H, dtype=np.float64), np.arange(W, dtype=np.float64), indexing="ij")
    rx = (0.25 + 0.1 * np.sin(2 * np.pi * y / H)).astype(np.float32)
    ry = (0.25 + 0.1 * np.sin(2 * np.pi * x / W)).astype(np.float32)
    m.field_dx = np.stack([D, D]); m.field_dy = np.stack([D, D])
    m.field_rx = np.stack([rx, rx]); m.field_ry = np.stack([ry, ry])
    return m


def _ref_many(m, init, R, seed_base, max_snaps):
    desc, keep = m.to_desc()
    block = m.num_species * m.area
    snaps = np.zeros((R, max_snaps, block), np.int32)
    f = [np.ascontiguousarray(a, np.float32) for a in (m.field_dx, m.field_dy, m.field_rx, m.field_ry)]
    oracle.orc().orc_ref_solve_many_snaps(oracle.model_ptr(desc), oracle.ptr(np.ascontiguousarray(init[0])), R,
                                          seed_base, *[oracle.ptr(a) for a in f], max_snaps, oracle.ptr(snaps))
    return snaps


def test_inhomogeneous_replay_matches_reference_statistics():
    """Drift-diffusion: the replay (binomial sweeps, Philox) and the reference-exact
    restatement of the inhomogeneous event loop (one Threefry uniform per particle and
    sweep, the reference's time steps and seeding) agree in per-cell mean and variance
    at both output windows."""
    from scipy import stats
    m = _c3_shaped()
    desc, keep = m.to_desc()
    R = 1500
    init = oracle.init_poisson(m.width, m.height, 2, 1, 11, [30.0, 30.0])
    st, rs, rt, rsteps, _ = oracle.rep_solve(desc, np.repeat(init, R, axis=0), R, 77, 8)
    ref = _ref_many(m, init, R, 5000, 3)
    assert rs.shape[0] == 3
    for w in (1, 2):
        a = rs[w].reshape(R, -1).astype(np.float64)
        b = ref[:, w].astype(np.float64)
        se = np.sqrt(a.var(0, ddof=1) / R + b.var(0, ddof=1) / R) + 1e-12
        z = np.abs(a.mean(0) - b.mean(0)) / se
        alpha = 1e-3 / z.size
        assert (z < stats.norm.isf(alpha / 2)).all(), (w, z.max())
        f = a.var(0, ddof=1) / np.maximum(b.var(0, ddof=1), 1e-12)
        lo, hi = stats.f.ppf(alpha / 2, R - 1, R - 1), stats.f.isf(alpha / 2, R - 1, R - 1)
        assert ((b.var(0) == 0) | ((f > lo) & (f < hi))).all(), w
