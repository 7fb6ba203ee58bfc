"""Model code compiled at run time (NVRTC) into the SSA and drift/diffusivity
kernels, as the reference generates its kernels from the model: custom propensity
laws and drift methods in code, checked bit for bit against the prebuilt kernels and
the oracle's replay, and model files in the reference's format end to end."""
import copy
import ctypes as C
import os

import numpy as np
import pytest

import oracle
from helpers import small_homog
from inchman_b200 import _lib, sbml
from inchman_b200.model import DiffusionModel

pytestmark = pytest.mark.gpu
MODELS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "models")


def _solve(m, init, R, seed, max_snaps=16):
    from inchman_b200.solver import Solver
    with Solver(m, realisations=R, seed=seed) as s:
        s.set_state(init)
        snaps, times, steps = s.solve(max_snapshots=max_snaps)
        return snaps, times, steps, s.status()


def _f(v):
    return repr(float(np.float32(v))) + "f"


def test_custom_laws_equal_to_mass_action_give_the_same_bits(gpgmp):
    m = small_homog(W=16, H=12, max_time=0.4)
    R, seed = 3, 99
    init = oracle.init_poisson(16, 12, 3, R, 4, [60.0, 40.0, 5.0])
    base = _solve(m, init, R, seed)
    mc = copy.deepcopy(m)
    mc.custom_laws = [f"(({_f(0.01)} * X(0)) * X(1))", f"({_f(0.1)} * X(2))"]
    got = _solve(mc, init, R, seed)
    assert got[2] == base[2] and np.array_equal(got[0], base[0]) and np.array_equal(got[3], base[3])


def test_custom_saturating_law_matches_replay(gpgmp):
    lm = sbml.load(os.path.join(MODELS, "saturating.xml"))
    m = lm.model
    R, seed = 2, 17
    init = m.initial_state(np.random.default_rng(1), R)
    snaps, times, steps, status = _solve(m, init, R, seed)
    f32 = np.float32

    def hz(r, x):
        s = f32(x[0])
        if r == 0:
            return (f32(40.0) * s) / (f32(25.0) + s)
        return f32(0.3) * s

    desc, keep = m.to_desc()
    cb = oracle.set_custom_hazard(hz)
    try:
        st, osn, ot, osteps, ostatus = oracle.rep_solve(desc, init, R, seed, 16)
    finally:
        oracle.set_custom_hazard(None)
    assert steps == osteps and np.array_equal(times, ot)
    assert np.array_equal(snaps, osn)
    assert snaps[-1][:, 1].sum() > 0          # the custom law produced P


def _inhom(W=16, method=_lib.DRIFT_ORNSTEIN_UHLENBECK, params=(1.0, 0.7, 0.5, 0.6, 0.7, 0.8, 0, 0)):
    m = DiffusionModel(width=W, height=W, physical_length=8.0, p0=0.1, max_time=0.4, output_interval=0.1,
                       solver=_lib.STOCHASTIC_INHOMOGENEOUS, drift_method=method, drift_params=params)
    m.add_species("A", 1.0).add_species("B", 1.0)
    m.add_reaction("ab", {"A": 1, "B": 1}, {}, 0.01)
    return m


@pytest.mark.parametrize("builtin,code", [
    ((_lib.DRIFT_ORNSTEIN_UHLENBECK, (1.0, 0.7, 0.5, 0.6, 0.7, 0.8, 0, 0)),
     "All->DiffusivityX = 1.0f; All->DiffusivityY = 0.7f;\n"
     "All->DriftX = -(0.5f * PhysicalX + 0.6f * PhysicalY);\nAll->DriftY = -(0.7f * PhysicalX + 0.8f * PhysicalY);"),
    ((_lib.DRIFT_MULTIPLICATIVE_NOISE, (0.5, 0.25, 0.1, 0.2, 0, 0, 0, 0)),
     "Real sx = PhysicalX + PhysicalModelWidth; Real sy = PhysicalY + PhysicalModelHeight;\n"
     "All->DiffusivityX = (0.5f * 0.5f) * (sx * sx) * 0.5f; All->DiffusivityY = (0.25f * 0.25f) * (sy * sy) * 0.5f;\n"
     "All->DriftX = 0.1f * sx; All->DriftY = 0.2f * sy;"),
])
def test_drift_code_matches_builtin_method(gpgmp, builtin, code):
    from inchman_b200.solver import Solver
    m = _inhom(method=builtin[0], params=builtin[1])
    mc = copy.deepcopy(m)
    mc.drift_method, mc.drift_code = _lib.DRIFT_CODE, code
    R, seed = 2, 5
    init = oracle.init_poisson(16, 16, 2, R, 9, [40.0, 30.0])
    with Solver(m, realisations=R, seed=seed) as a, Solver(mc, realisations=R, seed=seed) as b:
        assert [np.array_equal(x, y) for x, y in zip(a.timesteps(), b.timesteps())] == [True, True]
    base = _solve(m, init, R, seed)
    got = _solve(mc, init, R, seed)
    assert got[2] == base[2] and np.array_equal(got[0], base[0])


def test_model_file_end_to_end_matches_replay(gpgmp):
    """ab_drift.xml: mass-action laws and a drift method in code (species-specific
    drift), loaded and solved; the replay gets the same fields as arrays."""
    m = sbml.load(os.path.join(MODELS, "ab_drift.xml")).model
    R, seed = 2, 31
    init = m.initial_state(np.random.default_rng(3), R)
    snaps, times, steps, status = _solve(m, init, R, seed)
    mo = copy.deepcopy(m)
    mo.drift_method, mo.drift_code, mo.code_defines = _lib.DRIFT_FIELD, None, None
    shape = (2, m.height, m.width)
    f32 = np.float32
    mo.field_dx = np.full(shape, f32(1.0), np.float32)
    mo.field_dy = np.full(shape, f32(0.5), np.float32)
    mo.field_rx = np.stack([np.full(shape[1:], f32(0.4)), np.full(shape[1:], f32(-0.2))]).astype(np.float32)
    mo.field_ry = np.full(shape, f32(-0.1), np.float32)
    desc, keep = mo.to_desc()
    st, osn, ot, osteps, ostatus = oracle.rep_solve(desc, init, R, seed, 16)
    assert steps == osteps and np.array_equal(times, ot)
    assert np.array_equal(snaps, osn)


def test_code_that_does_not_compile_is_reported(gpgmp):
    from inchman_b200.solver import Solver
    m = small_homog(W=8, H=8, max_time=0.1)
    m.custom_laws = ["X(0) *** 2", None]
    with pytest.raises(_lib.GpgmpError) as e:
        Solver(m, realisations=1, seed=1)
    assert "does not compile" in str(e.value)
