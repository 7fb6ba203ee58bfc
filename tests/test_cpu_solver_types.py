"""The oracle's restatements of the remaining reference solver types
(DiffusionModel.h:46-56): alpha-QSS reaction windows (Deterministic.cl:240-522),
the inhomogeneous deterministic drift-diffusion sweeps (:71-136) and the FPE
discretisation of the stochastic inhomogeneous solver
(StochasticInhomogeneousDriftDiffusion.cl:124-129, 197-203) -- checked against
analytic solutions and invariants on the CPU."""
import ctypes as C

import numpy as np
import pytest

import oracle
from inchman_b200 import _lib
from inchman_b200.model import DiffusionModel


def _one_cell(solver, reactions, species):
    m = DiffusionModel(width=1, height=1, physical_length=1.0, max_time=1.0, solver=solver)
    for sp in species:
        m.add_species(sp, 0.0)
    for name, re, pr, k in reactions:
        m.add_reaction(name, re, pr, k)
    return m


@pytest.mark.parametrize("T", [0.1, 1.0, 5.0])
def test_aqss_linear_exchange_matches_analytic(T):
    """A <-> B (2, 1) from A = 10: A(t) = 10/3 + (20/3) exp(-3 t)."""
    m = _one_cell(_lib.DETERMINISTIC_AQSS, [("f", {"A": 1}, {"B": 1}, 2.0), ("b", {"B": 1}, {"A": 1}, 1.0)], "AB")
    desc, keep = m.to_desc()
    y = np.array([10.0, 0.0], np.float32)
    assert oracle.orc().orc_aqss_cell(oracle.model_ptr(desc), oracle.ptr(y), T, 0) == 0
    a = 10.0 / 3.0 + (20.0 / 3.0) * np.exp(-3.0 * T)
    assert abs(y[0] - a) / a < 5e-3 and abs(y[1] - (10 - a)) / (10 - a) < 5e-3, (y, a)


def test_aqss_gray_scott_kinetics_match_fine_rk4():
    F, k = 0.04, 0.06
    m = _one_cell(_lib.DETERMINISTIC_AQSS, [("r1", {"U": 1, "V": 2}, {"V": 3}, 1.0), ("r2", {"U": 1}, {}, F),
                                            ("r3", {"V": 1}, {}, F + k), ("r4", {}, {"U": 1}, F)], "UV")
    desc, keep = m.to_desc()
    y = np.array([0.5, 0.25], np.float32)
    assert oracle.orc().orc_aqss_cell(oracle.model_ptr(desc), oracle.ptr(y), 10.0, 0) == 0

    def f(x):
        u, v = x
        return np.array([-u * v * v - F * u + F, u * v * v - (F + k) * v])

    x, h = np.array([0.5, 0.25]), 1e-3
    for _ in range(10_000):
        k1 = f(x); k2 = f(x + h / 2 * k1); k3 = f(x + h / 2 * k2); k4 = f(x + h * k3)
        x = x + h / 6 * (k1 + 2 * k2 + 2 * k3 + k4)
    np.testing.assert_allclose(y, x, rtol=5e-3)


def test_aqss_reference_form_can_reject_forever():
    """The reference's predictor keeps the outer step's size on a retry
    (Deterministic.cl:381-387): a species growing from zero is rejected at every
    step size, so the window never ends (the reference's kernel would not return).
    The restatement stops after its pass limit and reports it."""
    m = _one_cell(_lib.DETERMINISTIC_AQSS, [("f", {"A": 1}, {"B": 1}, 2.0), ("b", {"B": 1}, {"A": 1}, 1.0)], "AB")
    desc, keep = m.to_desc()
    y = np.array([10.0, 0.0], np.float32)
    assert oracle.orc().orc_aqss_cell(oracle.model_ptr(desc), oracle.ptr(y), 1.0, 1) == 1


def _field_model(W, solver, D=0.5, rx=0.5, ry=0.0, reactions=()):
    m = DiffusionModel(width=W, height=W, physical_length=float(W), p0=0.1, max_time=10.0, output_interval=5.0,
                       solver=solver, drift_method=_lib.DRIFT_HOMOGENEOUS, drift_params=(D, D, rx, ry, 0, 0, 0, 0))
    m.add_species("A", 1.0)
    for name, re, pr, k in reactions:
        m.add_reaction(name, re, pr, k)
    return m


def test_det_sweep_keeps_a_uniform_state():
    m = _field_model(8, _lib.DETERMINISTIC_INHOMOGENEOUS_RK4)
    desc, keep = m.to_desc()
    s = np.full((1, 8, 8), 3.25, np.float32)
    out = np.zeros_like(s)
    D = np.full((1, 8, 8), 0.7, np.float32)
    r = np.full((1, 8, 8), -0.3, np.float32)
    for ydir in (0, 1):
        oracle.orc().orc_det_sweep(oracle.model_ptr(desc), oracle.ptr(s), oracle.ptr(out), 0, ydir, 0.05, 1.0,
                                   oracle.ptr(D), oracle.ptr(r))
        assert np.array_equal(out, s)


def _det_solve(m, state, max_snaps=8):
    desc, keep = m.to_desc()
    st = np.ascontiguousarray(state, np.float32).copy()
    snaps = np.zeros((max_snaps,) + st.shape, np.float32)
    times = np.zeros(max_snaps, np.float32)
    ns, steps = C.c_int(0), C.c_int64(0)
    rc = oracle.orc().orc_det_solve(oracle.model_ptr(desc), oracle.ptr(st), oracle.ptr(snaps), oracle.ptr(times),
                                    max_snaps, C.byref(ns), C.byref(steps))
    return rc, st, snaps[:min(ns.value, max_snaps)], times[:min(ns.value, max_snaps)], steps.value


@pytest.mark.parametrize("solver", [_lib.DETERMINISTIC_INHOMOGENEOUS_RK4, _lib.DETERMINISTIC_INHOMOGENEOUS_AQSS])
def test_det_inhomogeneous_drift_moves_the_centroid(solver):
    """Drift (0.5, 0) and D = 0.5 on a Gaussian bump: after t = 10 the centroid moved by
    about r t = 5 cells in x and not in y, and the bump widened."""
    W = 64
    m = _field_model(W, solver)
    y, x = np.mgrid[0:W, 0:W].astype(np.float64)
    g = np.exp(-((x - 24.0) ** 2 + (y - 32.0) ** 2) / (2 * 3.0 ** 2)).astype(np.float32)
    rc, st, snaps, times, steps = _det_solve(m, g[None] * 100.0)
    assert rc == 0 and steps > 0
    w = st[0].astype(np.float64)
    w = w / w.sum()
    cx, cy = (w * x).sum(), (w * y).sum()
    t = float(times[-1])
    assert abs(cx - 24.0 - 0.5 * t) < 0.1 * 0.5 * t, (cx, t)
    assert abs(cy - 32.0) < 0.05
    var_x = (w * (x - cx) ** 2).sum()
    assert var_x > 9.0


def test_det_inhomogeneous_reaction_windows_follow_flag():
    """Type 5 runs RK4 windows; flags bit 5 (no reactions, as the reference) leaves a
    pure decay model unchanged."""
    W = 8
    m = _field_model(W, _lib.DETERMINISTIC_INHOMOGENEOUS_RK4, rx=0.0, reactions=[("decay", {"A": 1}, {}, 0.1)])
    m.max_time = 2.0
    m.output_interval = 1.0
    state = np.full((1, W, W), 10.0, np.float32)
    _, st, _, times, _ = _det_solve(m, state)
    np.testing.assert_allclose(st, 10.0 * np.exp(-0.1 * float(times[-1])), rtol=1e-4)
    m.flags = _lib.FLAG_NO_INHOM_DET_REACTIONS
    _, st2, _, _, _ = _det_solve(m, state)
    np.testing.assert_allclose(st2, 10.0, rtol=1e-6)


def test_fpe_time_step_and_particle_conservation():
    from helpers import small_inhom
    m = small_inhom(W=12, H=12, max_time=0.3)
    m.solver = _lib.STOCHASTIC_INHOMOGENEOUS_FPE
    m.reactions = []
    desc, keep = m.to_desc()
    dx = m.physical_length / m.width
    stay = np.float32(1.0 - np.float64(np.float32(m.p0)))
    Dx = m.field_dx[0].astype(np.float32)
    rx = m.field_rx[0].astype(np.float32)
    want = (stay / np.float32(6.0) / (Dx / np.float32(dx * dx) + np.abs(rx) / np.float32(2.0 * dx))).min()
    Fdx, Fdy = np.zeros((2, 12, 12), np.float32), np.zeros((2, 12, 12), np.float32)
    Frx, Fry = np.zeros_like(Fdx), np.zeros_like(Fdx)
    oracle.orc().orc_rep_diffusivity_drift(oracle.model_ptr(desc), 0, oracle.ptr(Fdx), oracle.ptr(Fdy),
                                           oracle.ptr(Frx), oracle.ptr(Fry))
    got = oracle.orc().orc_rep_timestep(oracle.model_ptr(desc), 0, 0, oracle.ptr(Fdx), oracle.ptr(Frx))
    assert abs(got - want) <= 1e-6 * want, (got, want)
    init = oracle.init_poisson(12, 12, 2, 2, 11, [50.0, 50.0])
    st, snaps, times, steps, status = oracle.rep_solve(desc, init, 2, 5, 4)
    assert steps > 0 and np.array_equal(st.sum(axis=(2, 3)), init.sum(axis=(2, 3)))
    assert not np.array_equal(st, init)
