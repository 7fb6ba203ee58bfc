"""Pins the oracle's reference restatement against the reference itself.

oracle/_ref/libgpgmp_ref.so is the reference's own OpenCL kernel sources
(StochasticHomogeneousDiffusion.cl, StochasticInhomogeneousDriftDiffusion.cl,
Deterministic.cl) and vendored Random123 headers compiled unchanged for the CPU by
oracle/Makefile (`make ref`).  Every comparison here is bit-exact.
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
