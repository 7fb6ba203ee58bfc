"""GPU parity of the stochastic solvers: every kernel and the event loop are
compared bit-exactly with the oracle's CPU replay of the same Philox streams.
All calls go through the C ABI (libgpgmp_b200.so)."""
import numpy as np
import pytest

import oracle
from helpers import small_homog, small_inhom

pytestmark = pytest.mark.gpu


def _solver(m, R, seed, **kw):
    from inchman_b200.solver import Solver
    return Solver(m, realisations=R, seed=seed, **kw)


def test_init_poisson_bit_exact(gpgmp):
    m = small_homog(W=17, H=9)
    R, seed = 3, 77
    s = _solver(m, R, seed)
    lam = [100.0, 40.0, 0.0]
    s.init_poisson(lam)
    got = s.get_state()
    want = oracle.init_poisson(m.width, m.height, m.num_species, R, seed, lam)
    assert np.array_equal(got, want)
    assert abs(got[:, 0].mean() - 100.0) < 2.0


@pytest.mark.parametrize("window", [0.0, 1.0 / 60.0, 0.37])
def test_ssa_window_bit_exact(gpgmp, window):
    m = small_homog(W=20, H=12)
    desc, keep = m.to_desc()
    R, seed = 2, 1234
    rng = np.random.default_rng(1)
    st = rng.integers(0, 150, size=(R, m.num_species, m.height, m.width)).astype(np.int32)
    s = _solver(m, R, seed)
    s.set_state(st)
    assert s.do_reactions(window, 640) == 641
    got = s.get_state()
    want = st.copy()
    status = np.zeros(R, np.int32)
    oracle.orc().orc_rep_ssa(oracle.model_ptr(desc), oracle.ptr(want), R, seed, 640, window, oracle.ptr(status))
    assert np.array_equal(got, want)
    assert (s.status() == status).all()


@pytest.mark.parametrize("bmask,source", [((0, 0, 0, 0), (0, 0, 0, 0)), ((1, 1, 1, 1), (0, 0, 0, 0)),
                                          ((0, 1, 0, 1), (5, 3, 0, 2))])
def test_homogeneous_diffusion_bit_exact(gpgmp, bmask, source):
    m = small_homog(W=45, H=37, bmask=bmask, source=source)
    desc, keep = m.to_desc()
    R, seed = 2, 99
    rng = np.random.default_rng(2)
    st = rng.integers(0, 400, size=(R, m.num_species, m.height, m.width)).astype(np.int32)
    st[0, 1, 3, 4] = 5000  # exercise the binomial four-way split (more than 64 movers)
    s = _solver(m, R, seed)
    s.set_state(st)
    want = st.copy()
    for sp in (0, 2, 1):
        s.diffuse(sp, 10.0, 64 * 7)
        oracle.orc().orc_rep_homog_diffuse(oracle.model_ptr(desc), oracle.ptr(want), R, seed, sp, 64 * 7)
    got = s.get_state()
    assert np.array_equal(got, want)
    if bmask == (0, 0, 0, 0) and source == (0, 0, 0, 0):
        assert (got.sum(axis=(2, 3)) == st.sum(axis=(2, 3))).all()  # reflecting walls conserve


def test_inhomogeneous_timesteps_and_sweeps_bit_exact(gpgmp):
    m = small_inhom(W=40, H=40)
    desc, keep = m.to_desc()
    R, seed = 2, 5
    s = _solver(m, R, seed)
    dtx, dty = s.timesteps()
    fields = [np.ascontiguousarray(f, dtype=np.float32) for f in (m.field_dx, m.field_dy, m.field_rx, m.field_ry)]
    for sp in range(2):
        ox = oracle.orc().orc_rep_timestep(oracle.model_ptr(desc), sp, 0, oracle.ptr(fields[0]), oracle.ptr(fields[2]))
        oy = oracle.orc().orc_rep_timestep(oracle.model_ptr(desc), sp, 1, oracle.ptr(fields[1]), oracle.ptr(fields[3]))
        assert dtx[sp] == np.float32(ox) and dty[sp] == np.float32(oy)
    rng = np.random.default_rng(4)
    st = rng.integers(0, 300, size=(R, 2, m.height, m.width)).astype(np.int32)
    s.set_state(st)
    want = st.copy()
    seed_in = 128
    out = s.diffuse(0, float(max(dtx[0], dty[0])), seed_in)
    sd = seed_in
    oracle.orc().orc_rep_inhomog_sweep(oracle.model_ptr(desc), oracle.ptr(want), R, seed, 0, 0, sd, float(dtx[0]),
                                       oracle.ptr(fields[0]), oracle.ptr(fields[2]))
    sd += 1
    oracle.orc().orc_rep_inhomog_sweep(oracle.model_ptr(desc), oracle.ptr(want), R, seed, 0, 1, sd, float(dty[0]),
                                       oracle.ptr(fields[1]), oracle.ptr(fields[3]))
    sd += 1
    assert out == sd
    assert np.array_equal(s.get_state(), want)


@pytest.mark.parametrize("kind", ["homogeneous", "inhomogeneous"])
def test_full_event_loop_bit_exact(gpgmp, kind):
    if kind == "homogeneous":
        m = small_homog(W=24, H=20, max_time=0.6)
    else:
        m = small_inhom(W=24, H=24, max_time=0.12)
    desc, keep = m.to_desc()
    R, seed = 3, 4321
    lam = [s.initial for s in m.species]
    init = oracle.init_poisson(m.width, m.height, m.num_species, R, seed, lam)
    s = _solver(m, R, seed)
    s.set_state(init)
    snaps, times, steps = s.solve(max_snapshots=16)
    _, osnaps, otimes, osteps, ostatus = oracle.rep_solve(desc, init, R, seed, 16)
    assert steps == osteps
    assert np.array_equal(times, otimes)
    assert np.array_equal(snaps, osnaps)
    assert (s.status() == ostatus).all()


def test_plain_sync_each_launch_matches_async(gpgmp):
    m = small_homog(W=16, H=16, max_time=0.3)
    R, seed = 1, 11
    a = _solver(m, R, seed)
    b = _solver(m, R, seed, sync_each_launch=True)
    a.init_poisson([60, 40, 5])
    b.init_poisson([60, 40, 5])
    sa = a.solve(max_snapshots=8)
    sb = b.solve(max_snapshots=8)
    assert np.array_equal(sa[0], sb[0]) and sa[2] == sb[2]


def test_deterministic_rk4_matches_oracle(gpgmp):
    from inchman_b200 import _lib
    m = small_homog(W=16, H=16, max_time=0.05)
    m.solver = _lib.DETERMINISTIC_RK4
    m.output_interval = 0.02
    desc, keep = m.to_desc()
    rng = np.random.default_rng(9)
    st = (rng.random((1, m.num_species, m.height, m.width)) * 50).astype(np.float32)
    s = _solver(m, 1, 0)
    s.set_state(st)
    snaps, times, steps = s.solve(max_snapshots=16)
    want = st[0].copy()
    osnaps = np.zeros((16,) + want.shape, np.float32)
    otimes = np.zeros(16, np.float32)
    import ctypes as C
    ns, osteps = C.c_int(0), C.c_int64(0)
    oracle.orc().orc_det_solve(oracle.model_ptr(desc), oracle.ptr(want), oracle.ptr(osnaps), oracle.ptr(otimes), 16,
                               C.byref(ns), C.byref(osteps))
    assert steps == osteps.value
    n = ns.value
    np.testing.assert_allclose(snaps[:n, 0], osnaps[:n], rtol=1e-5, atol=1e-5)
