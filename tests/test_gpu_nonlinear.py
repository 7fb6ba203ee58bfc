"""Nonlinear drift/diffusivity methods (InhomogeneousSolver.cpp:288-335, helpers.cl:18-21):
after every sweep the method is evaluated again on the state and time then -- with the
moments (MeanX) after an x sweep -- and the next time step of that direction follows.
Checked bit for bit against the oracle's sweep with the method restated in numpy
(float32, no fused multiply-add, as the run-time compiled method is built)."""
import ctypes as C

import numpy as np
import pytest

import oracle
from inchman_b200 import _lib
from inchman_b200.model import DiffusionModel
from inchman_b200.solver import Solver

CODE = ("All->DiffusivityX = 0.2f + 0.01f * All->State; All->DiffusivityY = 0.3f; "
        "All->DriftX = -0.05f * All->MeanX; All->DriftY = 0.0f;")


def mean_x(plane, W, L):
    """MeanX (helpers.cl:18-21) from the exact sums, in float32."""
    f = np.float32
    n = plane.sum()
    mx = (plane * np.arange(W)[None, :]).sum()
    return f(L) / f(W) * (f(np.float32(mx) / np.float32(n)) - f(W) / f(2.0))


def method(plane, meanx):
    """The method above per cell, in float32 as the device evaluates it."""
    f = np.float32
    st = plane.astype(np.float32)
    Dx = f(0.2) + f(0.01) * st
    Dy = np.full_like(st, f(0.3))
    rx = np.full_like(st, f(-0.05) * meanx)
    ry = np.zeros_like(st)
    return [a.astype(np.float32).reshape(-1) for a in (Dx, Dy, rx, ry)]


def _model(W):
    m = DiffusionModel(width=W, height=W, physical_length=float(W), solver=_lib.STOCHASTIC_INHOMOGENEOUS)
    m.add_species("A", 0.0)
    m.drift_method = _lib.DRIFT_CODE
    m.drift_code = CODE
    m.code_defines = "#define A SP(0)"
    m.flags = _lib.FLAG_NONLINEAR | _lib.FLAG_COMPUTE_MOMENTS
    m.max_time = 1.0
    m.output_interval = 1.0
    return m


@pytest.mark.gpu
def test_nonlinear_method_is_evaluated_after_every_sweep(gpgmp):
    W, seed, step = 16, 13, 50
    m = _model(W)
    rng = np.random.default_rng(2)
    st0 = np.zeros((1, 1, W, W), np.int32)
    st0[0, 0] = rng.poisson(20.0, (W, W))
    st0[0, 0, :, :4] += 30                            # lopsided, so MeanX is not 0
    with Solver(m, realisations=1, seed=seed) as s:
        s.set_state(st0)
        dtx0, dty0 = s.timesteps()
        t = float(max(dtx0[0], dty0[0]))
        assert s.diffuse(0, t, step) == step + 2
        g = s.get_state()
        dtx1, dty1 = s.timesteps()
    d, keep = m.to_desc()
    o = oracle.orc()

    def ts(D, r):
        return o.orc_rep_timestep(C.byref(d), 0, 0, oracle.ptr(D), oracle.ptr(r))

    L = m.physical_length
    f0 = method(st0[0, 0], mean_x(st0[0, 0], W, L))
    assert dtx0[0] == np.float32(ts(f0[0], f0[2])) and dty0[0] == np.float32(ts(f0[1], f0[3]))
    state = st0.copy()
    o.orc_rep_inhomog_sweep(C.byref(d), oracle.ptr(state), 1, seed, 0, 0, step, float(dtx0[0]), oracle.ptr(f0[0]),
                            oracle.ptr(f0[2]))
    mx1 = mean_x(state[0, 0], W, L)                   # the moments follow x sweeps only
    f1 = method(state[0, 0], mx1)
    o.orc_rep_inhomog_sweep(C.byref(d), oracle.ptr(state), 1, seed, 0, 1, step + 1, float(dty0[0]),
                            oracle.ptr(f1[1]), oracle.ptr(f1[3]))
    f2 = method(state[0, 0], mx1)
    assert np.array_equal(g, state)
    assert dtx1[0] == np.float32(ts(f1[0], f1[2]))
    assert dty1[0] == np.float32(ts(f2[1], f2[3]))


def test_nonlinear_methods_need_one_realisation(gpgmp):
    """Rejected before any device work (runs without a GPU)."""
    m = _model(8)
    d, keep = m.to_desc()
    h = C.c_void_p()
    rc = _lib.lib().gpgmp_solver_create(C.byref(d), 2, 0, 0, C.byref(h))
    assert rc == 4 and not h.value                    # GPGMP_ERR_UNSUPPORTED
