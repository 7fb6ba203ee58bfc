"""Field parameters (DiffusionModel.cpp:402-404, Solver.cpp:88-101,269-272,583-653,
736-747): per-cell values the drift method reads, updated by the setField method every
step; checked bit for bit against the method restated in numpy (float32) and the
oracle's time step."""
import ctypes as C

import numpy as np
import pytest

import oracle
from inchman_b200 import _lib
from inchman_b200.model import DiffusionModel
from inchman_b200.solver import Solver

DEFINES = "#define conc F(0)\n#define A SP(0)"
DRIFT = "All->DiffusivityX = 0.1f + conc; All->DiffusivityY = 0.2f; All->DriftX = 0.0f; All->DriftY = 0.0f;"
SET_FIELD = "#undef A\n#define A X(0)\nconc = conc + deltat; A = A + 1;"


def _model(W, values, set_field=SET_FIELD):
    m = DiffusionModel(width=W, height=W, physical_length=float(W), solver=_lib.STOCHASTIC_INHOMOGENEOUS)
    m.add_species("A", 0.0)
    m.drift_method = _lib.DRIFT_CODE
    m.drift_code = DRIFT
    m.code_defines = DEFINES
    m.field_names = ["conc"]
    m.field_values = values
    m.set_field_code = set_field
    m.max_time = 1.0
    m.output_interval = 1.0
    return m


@pytest.mark.gpu
def test_fields_drive_the_drift_method_and_the_set_field_method_updates_them(gpgmp):
    W = 12
    rng = np.random.default_rng(4)
    conc = rng.uniform(0.0, 0.5, (1, W, W)).astype(np.float32)
    m = _model(W, conc)
    st = rng.poisson(6.0, (1, 1, W, W)).astype(np.int32)
    d, keep = m.to_desc()
    o = oracle.orc()

    def dt_x(c):
        D = (np.float32(0.1) + c.reshape(-1)).astype(np.float32)
        r = np.zeros_like(D)
        return np.float32(o.orc_rep_timestep(C.byref(d), 0, 0, oracle.ptr(D), oracle.ptr(r)))

    with Solver(m, realisations=1, seed=1) as s:
        s.set_state(st)
        assert np.array_equal(s.get_fields(), conc)
        assert s.timesteps()[0][0] == dt_x(conc)
        s.update_fields(0.5, 0.0)
        assert np.array_equal(s.get_fields(), (conc + np.float32(0.5)).astype(np.float32))
        assert np.array_equal(s.get_state(), st + 1)
        new = np.full((1, W, W), 0.05, np.float32)
        s.set_fields(new)
        assert s.timesteps()[0][0] == dt_x(new)


def test_set_field_method_needs_one_realisation(gpgmp):
    """Rejected before any device work (runs without a GPU)."""
    m = _model(8, None)
    d, keep = m.to_desc()
    h = C.c_void_p()
    rc = _lib.lib().gpgmp_solver_create(C.byref(d), 2, 0, 0, C.byref(h))
    assert rc == 4 and not h.value                    # GPGMP_ERR_UNSUPPORTED
