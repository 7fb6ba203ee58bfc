"""Pins the oracle's reference restatement against the reference itself.

oracle/_ref/libgpgmp_ref.so is the reference's own OpenCL kernel sources
(StochasticHomogeneousDiffusion.cl, StochasticInhomogeneousDriftDiffusion.cl,
Deterministic.cl) and vendored Random123 headers compiled unchanged for the CPU by
oracle/Makefile (`make ref`), plus the reference's SSA and RK4 templates (Gillespie.cl,
Deterministic.cl) with their generator markers filled for fixed test models as
Solver.cpp:778-959 fills them (oracle/ref/gen_models.py).  Every comparison here is
bit-exact.
"""
import ctypes as C

import numpy as np
import pytest

import oracle
from helpers import small_homog, small_inhom

pytestmark = pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built (needs the reference sources)")


def _set_model(m):
    bm = np.array(m.boundary_mask, dtype=np.int32)
    oracle.ref().gref_set_model(m.width, m.height, m.num_species, m.physical_length, m.p0, oracle.ptr(bm))


def test_threefry_and_philox_match_vendored_random123():
    rng = np.random.default_rng(0)
    o, r = oracle.orc(), oracle.ref()
    for _ in range(500):
        key = rng.integers(0, 2**32, 2, dtype=np.uint32)
        c2 = rng.integers(0, 2**32, 2, dtype=np.uint32)
        a, b = np.zeros(2, np.uint32), np.zeros(2, np.uint32)
        o.orc_threefry2x32_20(oracle.ptr(c2), oracle.ptr(key), oracle.ptr(a))
        r.gref_threefry2x32(oracle.ptr(c2), oracle.ptr(key), oracle.ptr(b))
        assert (a == b).all()
        c4 = rng.integers(0, 2**32, 4, dtype=np.uint32)
        a4, b4 = np.zeros(4, np.uint32), np.zeros(4, np.uint32)
        o.orc_philox4x32_10(oracle.ptr(c4), oracle.ptr(key), oracle.ptr(a4))
        r.gref_philox4x32(oracle.ptr(c4), oracle.ptr(key), oracle.ptr(b4))
        assert (a4 == b4).all()


@pytest.mark.parametrize("bmask", [(0, 0, 0, 0), (1, 1, 1, 1), (1, 0, 0, 1)])
@pytest.mark.parametrize("species", [0, 2])
def test_homogeneous_diffusion_matches_reference_kernels(bmask, species):
    m = small_homog(W=13, H=11, bmask=bmask)
    desc, keep = m.to_desc()
    _set_model(m)
    rng = np.random.default_rng(species + 10 * bmask[0])
    st = rng.integers(0, 300, size=(m.num_species, m.height, m.width)).astype(np.int32)
    st[0, 0, 0] = 0
    a, b = st.copy(), st.copy()
    lost_a = np.zeros(4 * m.area, np.int32)
    lost_b = np.zeros(4 * m.area, np.int32)
    for seed in (0, 12345, -7):
        oracle.orc().orc_ref_homog_diffuse(oracle.model_ptr(desc), oracle.ptr(a), species, seed, oracle.ptr(lost_a))
        oracle.ref().gref_homog_diffuse(oracle.ptr(b), oracle.ptr(lost_b), seed, species)
        assert np.array_equal(a, b)
        assert np.array_equal(lost_a, lost_b)


@pytest.mark.parametrize("boundary", [0, 1, 2, 3])
def test_source_boundary_matches_reference_kernel(boundary):
    m = small_homog(W=12, H=12)
    desc, keep = m.to_desc()
    _set_model(m)
    st = np.zeros((m.num_species, m.height, m.width), np.int32)
    a, b = st.copy(), st.copy()
    oracle.orc().orc_ref_source_boundary(oracle.model_ptr(desc), oracle.ptr(a), 1, 99, boundary, 77)
    oracle.ref().gref_source_boundary(oracle.ptr(b), 99, 1, boundary, 77)
    assert np.array_equal(a, b) and a.sum() > 0


@pytest.mark.parametrize("sweep_y", [0, 1])
def test_inhomogeneous_sweep_matches_reference_kernels(sweep_y):
    m = small_inhom(W=16, H=16)
    m.boundary_mask = (0, 1, 1, 0)
    desc, keep = m.to_desc()
    _set_model(m)
    rng = np.random.default_rng(3)
    st = rng.integers(0, 200, size=(m.num_species, m.height, m.width)).astype(np.int32)
    a, b = st.copy(), st.copy()
    la, lb = np.zeros(4 * m.area, np.int32), np.zeros(4 * m.area, np.int32)
    fields = [np.ascontiguousarray(f, dtype=np.float32) for f in (m.field_dx, m.field_dy, m.field_rx, m.field_ry)]
    fp = [oracle.ptr(f) for f in fields]
    for species in (0, 1):
        oracle.orc().orc_ref_inhomog_diffuse(oracle.model_ptr(desc), oracle.ptr(a), species, 5, 0.02, sweep_y,
                                             *fp, oracle.ptr(la))
        oracle.ref().gref_inhomog_diffuse(oracle.ptr(b), *fp, oracle.ptr(lb), 5, species, 0.02, sweep_y)
        assert np.array_equal(a, b)


@pytest.mark.parametrize("sweep_y", [0, 1])
def test_timestep_matches_reference_kernel(sweep_y):
    m = small_inhom(W=16, H=16)
    desc, keep = m.to_desc()
    _set_model(m)
    fields = [np.ascontiguousarray(f, dtype=np.float32) for f in (m.field_dx, m.field_dy, m.field_rx, m.field_ry)]
    # exercise the zero-drift and zero-diffusivity branches too
    fields[2][0, 0, :3] = 0.0
    fields[3][0, 0, :3] = 0.0
    fields[0][0, 1, :2] = 0.0
    fields[1][0, 1, :2] = 0.0
    fp = [oracle.ptr(f) for f in fields]
    per_a = np.zeros(m.area, np.float32)
    per_b = np.zeros(m.area, np.float32)
    best = oracle.orc().orc_ref_timestep(oracle.model_ptr(desc), 0, sweep_y, *fp, oracle.ptr(per_a))
    oracle.ref().gref_timestep_cells(*fp, 0, sweep_y, oracle.ptr(per_b))
    np.testing.assert_array_equal(per_a, per_b)
    assert best == per_b.min()


def test_deterministic_stencil_matches_reference_kernel():
    m = small_homog(W=10, H=10)
    desc, keep = m.to_desc()
    _set_model(m)
    rng = np.random.default_rng(5)
    st = rng.random((m.num_species, m.height, m.width)).astype(np.float32)
    a = st.copy()
    out = np.zeros_like(a)
    D = np.array([s.diffusion for s in m.species], np.float32)
    oracle.orc().orc_ref_det_diffuse(oracle.model_ptr(desc), oracle.ptr(st), oracle.ptr(out), 0.01, 1)
    oracle.ref().gref_det_diffuse_inplace(oracle.ptr(a), oracle.ptr(D), 0.01)
    np.testing.assert_array_equal(out, a)


def _model(species, reactions, W=9, H=7, solver=None):
    """A DiffusionModel matching one of oracle/ref/gen_models.py's test models."""
    from inchman_b200 import _lib
    from inchman_b200.model import DiffusionModel
    m = DiffusionModel(width=W, height=H, physical_length=float(W), p0=0.1, max_time=1.0, output_interval=1.0,
                       solver=_lib.STOCHASTIC_HOMOGENEOUS if solver is None else solver)
    for sp in species:
        m.add_species(sp, 1.0)
    for rid, re_, pr, rate, regions in reactions:
        m.add_reaction(rid, re_, pr, rate, regions=regions)
    return m


_LEFT = [(0, 0, 3, 6)]
_SPOT = [(5, 2, 6, 3), (8, 6, 8, 6)]
SSA_MODELS = {
    "abc": (["A", "B", "C"], [("bind", {"A": 1, "B": 1}, {"C": 1}, 0.01, None),
                              ("unbind", {"C": 1}, {"A": 1, "B": 1}, 0.1, None)]),
    "dimer": (["A", "B"], [("dim", {"A": 2}, {"B": 1}, 0.005, None), ("split", {"B": 1}, {"A": 2}, 0.2, None),
                           ("src", {}, {"A": 1}, 3.0, None)]),
    "abcloc": (["A", "B", "C"], [("bind", {"A": 1, "B": 1}, {"C": 1}, 0.01, _LEFT),
                                 ("unbind", {"C": 1}, {"A": 1, "B": 1}, 0.1, None),
                                 ("make", {}, {"C": 1}, 2.5, _SPOT)]),
}


def _float_mask(m):
    mk = m.reaction_mask()
    if mk is None:
        return None
    return np.ascontiguousarray(mk.astype(np.float32))


@pytest.mark.parametrize("name", ["abc", "dimer", "abcloc"])
@pytest.mark.parametrize("deltat", [1.0 / 60.0, 0.4])
def test_ssa_restatement_matches_reference_gillespie_kernel(name, deltat):
    """orc_ref_gillespie against performGillespie (Gillespie.cl) generated for the
    same model: hazards in double from the printed rates, the cumulative-hazard
    masks, the mask image of localised reactions, Threefry keyed per cell."""
    sp, rx = SSA_MODELS[name]
    m = _model(sp, rx)
    desc, keep = m.to_desc()
    _set_model(m)
    rng = np.random.default_rng(len(name))
    mask = _float_mask(m)
    fn = getattr(oracle.ref(), f"gref_ssa_{name}")
    for seed in (0, 77, -5):
        st = rng.integers(0, 150, size=(m.num_species, m.height, m.width)).astype(np.int32)
        st[:, 0, 0] = 0                 # a cell with no reactions possible except sources
        a, b = st.copy(), st.copy()
        oracle.orc().orc_ref_gillespie(oracle.model_ptr(desc), oracle.ptr(a), seed, deltat)
        fn(oracle.ptr(b), seed, deltat, oracle.ptr(mask))
        assert np.array_equal(a, b), (seed, int((a != b).sum()))
        assert not np.array_equal(a, st)
    if mask is not None:                 # the localised reactions are off somewhere
        assert mask[0].any() and not mask[0].all() and not mask[2].all()


GS_REACTIONS = [("r1", {"U": 1, "V": 2}, {"V": 3}, 1.0), ("r2", {"U": 1}, {}, 0.04), ("r3", {"V": 1}, {}, 0.1),
                ("r4", {}, {"U": 1}, 0.04)]


@pytest.mark.parametrize("name,regions", [("gs", [None] * 4), ("gsloc", [_LEFT, None, _SPOT, None])])
@pytest.mark.parametrize("deltat", [0.01, 1.0])
def test_rk4_restatement_matches_reference_rk4_kernel(name, regions, deltat):
    """orc_ref_rk4 against deterministic_performReaction_rk4 (Deterministic.cl) with
    the right-hand side Solver.cpp:922-959 generates for the Gray-Scott network
    (GrayScottModel.cpp:14-60): 20 RK4 substeps, double literals, clamp at 0."""
    from inchman_b200 import _lib
    rx = [(r[0], r[1], r[2], r[3], g) for r, g in zip(GS_REACTIONS, regions)]
    m = _model(["U", "V"], rx, solver=_lib.DETERMINISTIC_RK4)
    desc, keep = m.to_desc()
    _set_model(m)
    rng = np.random.default_rng(3)
    st = np.stack([0.5 + 0.5 * rng.random((m.height, m.width)),
                   0.25 * rng.random((m.height, m.width))]).astype(np.float32)
    st[1, 0, 0] = 0.0
    a, b = st.copy(), st.copy()
    mask = _float_mask(m)
    for _ in range(3):
        oracle.orc().orc_ref_rk4(oracle.model_ptr(desc), oracle.ptr(a), deltat)
        getattr(oracle.ref(), f"gref_rk4_{name}")(oracle.ptr(b), deltat, oracle.ptr(mask))
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), int((a != b).sum())
    assert not np.array_equal(a, st)
