"""Localised reactions on the GPU (Reaction::addCompartment / reactionMask,
Reaction.cpp:209-235; the mask image of Solver.cpp:352-390 multiplied into the
hazards, Solver.cpp:852-854, and into the deterministic right-hand side, :946-948).

Every stochastic case is bit-exact against the oracle's replay with the same masks;
the deterministic ones match the oracle's RK4 / alpha-QSS within the tolerances of
the unlocalised tests.  All calls go through the C ABI."""
import ctypes as C
import os

import numpy as np
import pytest

import oracle
from inchman_b200 import _lib, sbml
from inchman_b200.model import DiffusionModel

pytestmark = pytest.mark.gpu
MODELS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "models")


def _gpu_solve(m, state, R, seed=0, max_snaps=16):
    from inchman_b200.solver import Solver
    with Solver(m, realisations=R, seed=seed) as s:
        s.set_state(state)
        snaps, times, steps = s.solve(max_snapshots=max_snaps)
        return snaps, times, steps, s.status()


def _homog(W=16, H=12, max_time=0.5, extra=0):
    """A + B -> C only in the left block, C -> A + B only in a spot, 0 -> A only in the
    right column; `extra` more reactions (C -> C, localised to rows) push the network
    past the size at which the SSA keeps per-reaction hazards."""
    m = DiffusionModel(width=W, height=H, physical_length=float(W), p0=0.1, max_time=max_time, output_interval=0.1,
                       solver=_lib.STOCHASTIC_HOMOGENEOUS)
    m.add_species("A", 1.0).add_species("B", 0.7).add_species("C", 0.3)
    m.add_reaction("bind", {"A": 1, "B": 1}, {"C": 1}, 0.01, regions=[(0, 0, W // 2 - 1, H - 1)])
    m.add_reaction("unbind", {"C": 1}, {"A": 1, "B": 1}, 0.5, regions=[(W - 4, 2, W - 2, 4), (1, H - 3, 2, H - 1)])
    m.add_reaction("source", {}, {"A": 1}, 20.0, regions=[(W - 1, 0, W - 1, H - 1)])
    m.add_reaction("decay", {"B": 1}, {}, 0.05)
    for q in range(extra):
        m.add_reaction(f"x{q}", {"C": 1}, {"A": 1, "C": 1}, 0.02 * (q + 1), regions=[(0, q % H, W - 1, q % H)])
    return m


@pytest.mark.parametrize("extra", [0, 6])
def test_localised_homogeneous_bit_exact_against_replay(gpgmp, extra):
    m = _homog(extra=extra)
    assert m.reaction_mask() is not None and not m.reaction_mask().all()
    R, seed = 3, 2024
    init = oracle.init_poisson(m.width, m.height, 3, R, 11, [60.0, 50.0, 10.0])
    snaps, times, steps, status = _gpu_solve(m, init, R, seed)
    desc, keep = m.to_desc()
    _, osn, ot, osteps, ostatus = oracle.rep_solve(desc, init, R, seed, 16)
    assert steps == osteps and np.array_equal(times, ot)
    assert np.array_equal(snaps, osn)
    assert (status == ostatus).all()
    # the masks changed the run: without them the same seed gives other counts
    m2 = _homog(extra=extra)
    for r in m2.reactions:
        r.regions = []
    other, _, _, _ = _gpu_solve(m2, init, R, seed)
    assert not np.array_equal(other[-1], snaps[-1])


def test_reactions_fire_only_inside_their_regions(gpgmp):
    """One reaction window through doReactions: the counts of cells outside every
    region stay as they were, and a source adds only inside its region."""
    from inchman_b200.solver import Solver
    W = H = 12
    m = DiffusionModel(width=W, height=H, physical_length=float(W), p0=0.1, max_time=1.0, output_interval=0.5,
                       solver=_lib.STOCHASTIC_HOMOGENEOUS)
    m.add_species("A", 0.0).add_species("B", 0.0)
    m.add_reaction("conv", {"A": 1}, {"B": 1}, 2.0, regions=[(2, 3, 5, 7)])
    m.add_reaction("src", {}, {"B": 1}, 30.0, regions=[(9, 9, 10, 10), (0, 0, 0, 0)])
    mask = m.reaction_mask().astype(bool)
    init = np.full((2, 2, H, W), 40, np.int32)
    with Solver(m, realisations=2, seed=5) as s:
        s.set_state(init)
        assert s.do_reactions(1.0, 10) == 11
        fin = s.get_state()
        status = s.status()
    inside_conv, inside_src = mask[0], mask[1]
    assert (fin[:, 0][:, ~inside_conv] == 40).all()              # A converts only inside
    assert (fin[:, 0][:, inside_conv] < 40).all()
    untouched = ~inside_conv & ~inside_src
    assert (fin[:, 1][:, untouched] == 40).all()                 # B changes only in the regions
    assert (fin[:, 1][:, inside_src] > 40).all()
    desc, keep = m.to_desc()
    want = init.copy()
    oracle.orc().orc_rep_ssa(oracle.model_ptr(desc), oracle.ptr(want), 2, 5, 10, 1.0, None)
    assert np.array_equal(fin, want)
    assert (status == 0).all()


def test_localised_inhomogeneous_bit_exact_against_replay(gpgmp):
    W = 16
    m = DiffusionModel(width=W, height=W, physical_length=float(W), p0=0.1, max_time=0.3, output_interval=0.1,
                       solver=_lib.STOCHASTIC_INHOMOGENEOUS, drift_method=_lib.DRIFT_FIELD)
    m.add_species("X", 1.0).add_species("Y", 1.0)
    m.add_reaction("birth", {"X": 1}, {"X": 2}, 1.0, regions=[(0, 0, 7, 15)])
    m.add_reaction("predation", {"X": 1, "Y": 1}, {"Y": 2}, 0.005)
    m.add_reaction("death", {"Y": 1}, {}, 0.6, regions=[(4, 4, 11, 11)])
    rng = np.random.Generator(np.random.PCG64(3))
    D = rng.lognormal(0.0, 0.5, size=(W, W)).astype(np.float32)
    y, x = np.meshgrid(np.arange(W, dtype=np.float64), np.arange(W, dtype=np.float64), indexing="ij")
    rx = (0.3 * np.sin(2 * np.pi * y / W)).astype(np.float32)
    ry = (0.3 * np.cos(2 * np.pi * x / W)).astype(np.float32)
    m.field_dx = np.stack([D, D]); m.field_dy = np.stack([D, D])
    m.field_rx = np.stack([rx, rx]); m.field_ry = np.stack([ry, ry])
    R, seed = 2, 77
    init = oracle.init_poisson(W, W, 2, R, 5, [50.0, 50.0])
    snaps, times, steps, status = _gpu_solve(m, init, R, seed)
    desc, keep = m.to_desc()
    _, osn, ot, osteps, _ = oracle.rep_solve(desc, init, R, seed, 16)
    assert steps == osteps and np.array_equal(times, ot)
    assert np.array_equal(snaps, osn)


def test_localised_model_file_with_custom_law_matches_replay(gpgmp):
    """localised.xml: a source only in a spot, A + B -> C only on the left, a
    saturating (run-time compiled) law only on the right; loaded, solved, and
    compared with the replay given the same law as a callback."""
    lm = sbml.load(os.path.join(MODELS, "localised.xml"))
    m = lm.model
    assert m.custom_laws is not None and m.reaction_mask() is not None
    R, seed = 2, 41
    init = m.initial_state(np.random.default_rng(2), R)
    snaps, times, steps, status = _gpu_solve(m, init, R, seed)
    f32 = np.float32

    def hz(r, x):
        if r == 0:
            return f32(30.0)
        if r == 1:
            return (f32(0.02) * f32(x[0])) * f32(x[1])
        if r == 2:
            return f32(0.4) * f32(x[2])
        b = f32(x[1])
        return (f32(12.0) * b) / (f32(10.0) + b)

    desc, keep = m.to_desc()
    cb = oracle.set_custom_hazard(hz)
    try:
        _, osn, ot, osteps, _ = oracle.rep_solve(desc, init, R, seed, 16)
    finally:
        oracle.set_custom_hazard(None)
    assert steps == osteps and np.array_equal(times, ot)
    assert np.array_equal(snaps, osn)


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


@pytest.mark.parametrize("solver,rtol,atol", [(_lib.DETERMINISTIC_RK4, 1e-5, 1e-5),
                                              (_lib.DETERMINISTIC_AQSS, 1e-5, 1e-6)])
def test_localised_deterministic_matches_oracle(gpgmp, solver, rtol, atol):
    W = 8
    F, k = 0.04, 0.06
    m = DiffusionModel(width=W, height=W, physical_length=float(W), p0=0.1, max_time=1.0, output_interval=0.25,
                       solver=solver)
    m.add_species("U", 0.16).add_species("V", 0.08)
    m.add_reaction("r1", {"U": 1, "V": 2}, {"V": 3}, 1.0, regions=[(0, 0, 3, 7)])
    m.add_reaction("r2", {"U": 1}, {}, F)
    m.add_reaction("r3", {"V": 1}, {}, F + k, regions=[(2, 2, 5, 5)])
    m.add_reaction("r4", {}, {"U": 1}, F, regions=[(4, 0, 7, 7)])
    rng = np.random.default_rng(4)
    st = np.stack([0.5 + 0.1 * rng.random((W, W)), 0.25 + 0.1 * rng.random((W, W))])[None].astype(np.float32)
    snaps, times, steps, status = _gpu_solve(m, st, 1)
    rc, osn, ot, osteps = _orc_det(m, st[0])
    assert rc == 0 and steps == osteps and int(status[0]) == 0
    np.testing.assert_allclose(snaps[:, 0], osn, rtol=rtol, atol=atol)
    for r in m.reactions:
        r.regions = []
    other, _, _, _ = _gpu_solve(m, st, 1)
    assert np.abs(other[-1] - snaps[-1]).max() > 1e-3
