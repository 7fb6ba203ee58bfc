"""The remaining reference solver types on the GPU against the oracle:
stochastic_inhomogeneous_fpe (bit-exact replay), deterministic_homogeneous_aqss,
deterministic_inhomogeneous_RK4 and deterministic_inhomogeneous_aqss (sweeps and
alpha-QSS windows as the oracle restates them; RK4 windows to 1e-5 as for the
homogeneous RK4 solver)."""
import ctypes as C

import numpy as np
import pytest

import oracle
from helpers import small_inhom
from inchman_b200 import _lib
from inchman_b200.model import DiffusionModel

pytestmark = pytest.mark.gpu


def _gpu_solve(m, state, R, seed=0, max_snaps=16):
    from inchman_b200.solver import Solver
    with Solver(m, realisations=R, seed=seed) as s:
        s.set_state(state)
        snaps, times, steps = s.solve(max_snapshots=max_snaps)
        return snaps, times, steps, s.status()


def _orc_det(m, state, max_snaps=16):
    desc, keep = m.to_desc()
    st = np.ascontiguousarray(state, np.float32).copy()
    snaps = np.zeros((max_snaps,) + st.shape, np.float32)
    times = np.zeros(max_snaps, np.float32)
    ns, steps = C.c_int(0), C.c_int64(0)
    rc = oracle.orc().orc_det_solve(oracle.model_ptr(desc), oracle.ptr(st), oracle.ptr(snaps), oracle.ptr(times),
                                    max_snaps, C.byref(ns), C.byref(steps))
    n = min(ns.value, max_snaps)
    return rc, snaps[:n], times[:n], steps.value


def test_fpe_solver_matches_replay_bit_exact(gpgmp):
    m = small_inhom(W=16, H=16, max_time=0.3)
    m.solver = _lib.STOCHASTIC_INHOMOGENEOUS_FPE
    desc, keep = m.to_desc()
    R, seed = 3, 77
    init = oracle.init_poisson(16, 16, 2, R, 5, [50.0, 50.0])
    snaps, times, steps, status = _gpu_solve(m, init, R, seed)
    ost, osn, ot, osteps, ostatus = oracle.rep_solve(desc, init, R, seed, 16)
    assert steps == osteps and len(times) == len(ot)
    assert np.array_equal(snaps, osn) and np.array_equal(times, ot)
    assert np.array_equal(status, ostatus)


def _det_inhom_model(solver, W=16):
    m = small_inhom(W=W, H=W, max_time=0.6)
    m.solver = solver
    m.output_interval = 0.2
    return m


@pytest.mark.parametrize("solver,rtol", [(_lib.DETERMINISTIC_INHOMOGENEOUS_RK4, 1e-5),
                                         (_lib.DETERMINISTIC_INHOMOGENEOUS_AQSS, 1e-5)])
def test_det_inhomogeneous_matches_oracle(gpgmp, solver, rtol):
    m = _det_inhom_model(solver)
    rng = np.random.default_rng(3)
    st = (20.0 + 40.0 * rng.random((1, 2, 16, 16))).astype(np.float32)
    snaps, times, steps, status = _gpu_solve(m, st, 1)
    rc, osn, ot, osteps = _orc_det(m, st[0])
    assert rc == 0 and steps == osteps and int(status[0]) == 0
    np.testing.assert_array_equal(times, ot)
    np.testing.assert_allclose(snaps[:, 0], osn, rtol=rtol, atol=rtol)


def test_det_inhomogeneous_without_reactions_flag(gpgmp):
    m = _det_inhom_model(_lib.DETERMINISTIC_INHOMOGENEOUS_AQSS)
    m.flags = _lib.FLAG_NO_INHOM_DET_REACTIONS
    st = np.full((1, 2, 16, 16), 30.0, np.float32)
    snaps, times, steps, status = _gpu_solve(m, st, 1)
    rc, osn, ot, osteps = _orc_det(m, st[0])
    assert steps == osteps
    np.testing.assert_allclose(snaps[:, 0], osn, rtol=1e-6, atol=1e-5)


def _gs_kinetics_model(solver, W=8):
    F, k = 0.04, 0.06
    m = DiffusionModel(width=W, height=W, physical_length=float(W), p0=0.1, max_time=2.0, output_interval=0.5,
                       solver=solver)
    m.add_species("U", 0.16).add_species("V", 0.08)
    m.add_reaction("r1", {"U": 1, "V": 2}, {"V": 3}, 1.0)
    m.add_reaction("r2", {"U": 1}, {}, F)
    m.add_reaction("r3", {"V": 1}, {}, F + k)
    m.add_reaction("r4", {}, {"U": 1}, F)
    return m


def test_det_aqss_homogeneous_matches_oracle_and_rk4(gpgmp):
    m = _gs_kinetics_model(_lib.DETERMINISTIC_AQSS)
    rng = np.random.default_rng(4)
    st = np.stack([0.5 + 0.1 * rng.random((8, 8)), 0.25 + 0.1 * rng.random((8, 8))])[None].astype(np.float32)
    snaps, times, steps, status = _gpu_solve(m, st, 1)
    rc, osn, ot, osteps = _orc_det(m, st[0])
    assert rc == 0 and steps == osteps and int(status[0]) == 0
    np.testing.assert_allclose(snaps[:, 0], osn, rtol=1e-5, atol=1e-6)
    m.solver = _lib.DETERMINISTIC_RK4
    rk, _, _, _ = _gpu_solve(m, st, 1)
    np.testing.assert_allclose(snaps[-1], rk[-1], rtol=5e-3)


def test_aqss_reference_form_reports_the_stall(gpgmp):
    """The reference's alpha-QSS predictor can reject every step (a species growing
    from zero); the kernel stops at its pass limit and sets the realisation's
    GPGMP_SIM_EVENT_CAP bit instead of looping forever."""
    m = DiffusionModel(width=4, height=4, physical_length=4.0, p0=0.1, max_time=1.0, output_interval=1.0,
                       solver=_lib.DETERMINISTIC_AQSS, flags=_lib.FLAG_AQSS_LITERAL)
    m.add_species("A", 0.0).add_species("B", 0.0)
    m.add_reaction("f", {"A": 1}, {"B": 1}, 2.0)
    m.add_reaction("b", {"B": 1}, {"A": 1}, 1.0)
    st = np.zeros((1, 2, 4, 4), np.float32)
    st[0, 0] = 10.0
    snaps, times, steps, status = _gpu_solve(m, st, 1)
    assert int(status[0]) & _lib.SIM_EVENT_CAP
    m.flags = 0
    snaps, times, steps, status = _gpu_solve(m, st, 1)
    assert int(status[0]) == 0
    a = 10.0 / 3.0 + (20.0 / 3.0) * np.exp(-3.0 * float(times[-1]))
    np.testing.assert_allclose(snaps[-1, 0, 0], a, rtol=5e-3)
