"""Individual species inside the solver (IndividualSolver.cpp, IndividualSolver.cl;
InhomogeneousSolver.cpp:254-427): lists built from the counts, sweeps of individuals
with their own properties bit for bit against the oracle's restatement, model code
compiled at run time, reaction windows followed by the population bookkeeping and
the new-individuals method."""
import ctypes as C

import numpy as np
import pytest

import oracle
from inchman_b200 import _lib
from inchman_b200.model import DiffusionModel
from inchman_b200.solver import Solver


def _model(W=24, H=20, reactions=(), bmask=(0, 1, 0, 0), code=None, newborn=None):
    m = DiffusionModel(width=W, height=H, physical_length=float(W), solver=_lib.STOCHASTIC_INHOMOGENEOUS)
    m.add_species("A", 0.0, individual=True)
    m.add_species("B", 0.5)
    for rid, re, pr, k in reactions:
        m.add_reaction(rid, re, pr, k)
    m.boundary_mask = list(bmask)
    m.drift_method = _lib.DRIFT_HOMOGENEOUS
    m.drift_params = [0.5, 0.5, 0.0, 0.0] + [0.0] * 4
    if code is not None:
        m.drift_method = _lib.DRIFT_CODE
        m.drift_code = code
        m.code_defines = "#define A SP(0)\n#define B SP(1)"
    m.new_individuals_code = newborn
    m.max_time = 1.0
    m.output_interval = 1.0
    return m


def _state(m, R, seed, lam=(3.0, 4.0)):
    rng = np.random.default_rng(seed)
    return rng.poisson(lam, (R, m.height, m.width, 2)).transpose(0, 3, 1, 2).astype(np.int32).copy()


def _desc(m):
    d, keep = m.to_desc()
    return d, keep


@pytest.mark.gpu
def test_lists_are_built_from_the_counts(gpgmp):
    m = _model()
    R = 3
    st = _state(m, R, 1)
    with Solver(m, realisations=R, seed=5) as s:
        s.set_state(st)
        keys, ids, props = s.get_individuals(0)
        area = m.width * m.height
        assert len(keys) == int(st[:, 0].sum())
        assert np.all(np.diff(keys.astype(np.int64)) >= 0)
        assert np.array_equal(np.bincount(keys, minlength=R * area), st[:, 0].reshape(-1))
        assert np.array_equal(ids, np.arange(len(keys), dtype=np.uint32))    # ids in cell order
        assert np.all(props == 0.0)                                          # as the reference starts them
        assert np.array_equal(s.get_state(), st)


def _sweep_case(R=3, seed=7):
    m = _model()
    st = _state(m, R, seed)
    n = int(st[:, 0].sum())
    rng = np.random.default_rng(seed + 1)
    props = np.stack([rng.uniform(0.2, 1.0, n), rng.uniform(0.2, 1.0, n), rng.uniform(-0.3, 0.3, n),
                      rng.uniform(-0.3, 0.3, n)]).astype(np.float32)
    return m, st, props


@pytest.mark.gpu
def test_sweeps_match_the_oracle(gpgmp):
    R, seed = 3, 11
    m, st, props = _sweep_case(R)
    area = m.width * m.height
    with Solver(m, realisations=R, seed=seed) as s:
        s.set_state(st)
        s.set_individual_properties(0, props)
        dtx0, dty0 = s.timesteps()
        keys, ids, _ = s.get_individuals(0)
        nx = s.get_next_diffusion_time()
        t = float(max(dtx0[0], dty0[0]))
        step0 = 40
        after = s.diffuse(0, t, step0)
        assert after == step0 + 2                          # one seed per sweep
        g_state = s.get_state()
        g_keys, g_ids, g_props = s.get_individuals(0)
        dtx1, dty1 = s.timesteps()
    # the oracle: X then Y with the time steps the properties gave, new steps after each
    d, keep = m.to_desc()
    o_state = st.copy()
    k = keys.copy()
    i = ids.copy()
    n = len(k)
    fields = np.zeros(4 * R * area, np.float32)
    killed = np.zeros(max(1, n), np.uint32)
    nk = C.c_int64(0)
    o = oracle.orc()
    new_dt = []
    left = 0
    for dr, dt in ((0, dtx0[0]), (1, dty0[0])):
        left += o.orc_rep_ind_sweep(C.byref(d), oracle.ptr(o_state), R, seed, 0, dr, float(dt), step0 + dr,
                                    oracle.ptr(k), oracle.ptr(i), n, oracle.ptr(props), props.shape[1],
                                    oracle.ptr(fields))
        dx = m.physical_length / (m.width if dr == 0 else m.height)
        off = (0 if dr == 0 else 1) * R * area
        roff = (2 if dr == 0 else 3) * R * area
        new_dt.append(o.orc_rep_timestep_cells(oracle.ptr(fields[off:]), oracle.ptr(fields[roff:]), R * area,
                                               float(np.float32(dx))))
    # the list is sorted when read (once, after both sweeps)
    n = o.orc_rep_ind_sort(oracle.ptr(k), oracle.ptr(i), n, R * area, oracle.ptr(killed), C.byref(nk))
    assert nk.value == left > 0
    assert np.array_equal(g_state, o_state)
    assert np.array_equal(g_keys, k[:n]) and np.array_equal(g_ids, i[:n])
    assert len(g_keys) < len(keys)                      # some left through the absorbing wall (x+)
    assert dtx1[0] == np.float32(new_dt[0]) and dty1[0] == np.float32(new_dt[1])


@pytest.mark.gpu
def test_model_code_runs_per_individual(gpgmp):
    """A drift method in code that sets constants gives the same bits as the stored
    properties equal to those constants (run-time compiled vs prebuilt kernels)."""
    R, seed = 2, 3
    code = "All->DiffusivityX = 0.6f; All->DiffusivityY = 0.4f; All->DriftX = 0.2f; All->DriftY = -0.1f;"
    m_code = _model(code=code)
    m_plain = _model()
    st = _state(m_plain, R, 4)
    out = []
    for m, use_props in ((m_code, False), (m_plain, True)):
        with Solver(m, realisations=R, seed=seed) as s:
            s.set_state(st)
            if use_props:
                n = int(st[:, 0].sum())
                p = np.array([[0.6], [0.4], [0.2], [-0.1]], np.float32).repeat(n, axis=1)
                s.set_individual_properties(0, p)
            dtx, dty = s.timesteps()
            t = float(max(dtx[0], dty[0]))
            sd = 9
            for _ in range(3):
                sd = s.diffuse(0, t, sd)
                tx, ty = s.timesteps()
                t += float(max(tx[0], ty[0]))
            out.append((s.get_state(), s.get_individuals(0)[:2], s.timesteps()))
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1][0], out[1][1][0]) and np.array_equal(out[0][1][1], out[1][1][1])
    # the individual species' time steps (species B follows each model's own method)
    assert out[0][2][0][0] == out[1][2][0][0] and out[0][2][1][0] == out[1][2][1][0]


@pytest.mark.gpu
def test_reaction_windows_keep_the_lists_and_set_new_individuals(gpgmp):
    R, seed = 2, 21
    newborn = ("All->DiffusivityX = 0.25f + RANDOM; All->DiffusivityY = 2.0f; All->DriftX = -1.0f; "
               "All->DriftY = RANDOM;")
    m = _model(reactions=[("decay", {"A": 1}, {}, 0.4), ("make", {"B": 1}, {"A": 1, "B": 1}, 0.3)],
               bmask=(0, 0, 0, 0), newborn=newborn)
    st = _state(m, R, 8)
    area = m.width * m.height
    with Solver(m, realisations=R, seed=seed) as s:
        s.set_state(st)
        keys0, ids0, _ = s.get_individuals(0)
        old = set(ids0.tolist())
        step = 100
        nxt = s.do_reactions(0.5, step)
        assert nxt == step + 2                              # the window, then the bookkeeping
        state = s.get_state()
        keys, ids, props = s.get_individuals(0)
    assert np.all(np.diff(keys.astype(np.int64)) >= 0)
    assert np.array_equal(np.bincount(keys, minlength=R * area), state[:, 0].reshape(-1))
    assert len(np.unique(ids)) == len(ids)
    new = np.array([i not in old for i in ids.tolist()])
    assert new.any() and (~new).any()
    assert np.all(props[:, ~new] == 0.0)                    # survivors keep their properties
    # the new ones: the method with one Philox stream per individual (seed, realisation;
    # step seed of the bookkeeping, id, PH_NEWIND | species << 8)
    for j in np.flatnonzero(new)[:200]:
        r = int(keys[j]) // area
        u = np.zeros(4, np.uint32)
        oracle.orc().orc_philox_fill(seed, r, step + 1, int(ids[j]), 0x09000000, oracle.ptr(u), 2)
        u01 = (u[:2] >> 8).astype(np.float32) * np.float32(5.9604644775390625e-08)
        assert props[0, j] == np.float32(0.25) + u01[0]
        assert props[1, j] == 2.0 and props[2, j] == -1.0
        assert props[3, j] == u01[1]


def test_individual_species_need_an_inhomogeneous_solver(gpgmp):
    """Checked before any device work, so it runs without a GPU."""
    m = _model()
    m.solver = _lib.STOCHASTIC_HOMOGENEOUS
    d, keep = m.to_desc()
    h = C.c_void_p()
    rc = _lib.lib().gpgmp_solver_create(C.byref(d), 1, 0, 0, C.byref(h))
    assert rc == 4 and not h.value                      # GPGMP_ERR_UNSUPPORTED


@pytest.mark.gpu
def test_individual_sweeps_match_count_sweeps_in_distribution(gpgmp):
    """Individuals that all have the same D and r move like the molecules of the
    count-based sweep (a binomial number leaves each cell): per-cell means over 512
    realisations after 12 sweeps per direction agree within 5 standard errors, and so
    does the spread of the cloud."""
    W = 16
    R = 512
    D, r = 0.5, 0.15
    st = np.zeros((R, 2, W, W), np.int32)
    st[:, 0, 6:10, 6:10] = 25
    means, spreads = [], []
    for individual in (False, True):
        m = DiffusionModel(width=W, height=W, physical_length=float(W), solver=_lib.STOCHASTIC_INHOMOGENEOUS)
        m.add_species("A", 0.0, individual=individual)
        m.add_species("B", 0.0)
        m.drift_method = _lib.DRIFT_HOMOGENEOUS
        m.drift_params = [D, D, r, 0.0] + [0.0] * 4
        with Solver(m, realisations=R, seed=77) as s:
            s.set_state(st)
            if individual:
                n = int(st[:, 0].sum())
                s.set_individual_properties(0, np.array([[D], [D], [r], [0.0]], np.float32).repeat(n, axis=1))
            dtx, dty = s.timesteps()
            assert dtx[0] > 0 and dty[0] > 0
            sd = 1
            for k in range(12):
                t = float(max(dtx[0], dty[0]) * (k + 1))
                sd = s.diffuse(0, t, sd)
            a = s.get_state()[:, 0].astype(np.float64)
        means.append((a.mean(axis=0), a.var(axis=0)))
        x = np.arange(W)
        spreads.append(((a.sum(axis=1) * x).sum(axis=1) / a.sum(axis=(1, 2))).std())
    (m0, v0), (m1, v1) = means
    se = np.sqrt((v0 + v1) / R) + 1e-9
    assert np.all(np.abs(m0 - m1) <= 5 * se + 1e-6)
    assert abs(spreads[0] - spreads[1]) < 0.15 * spreads[0]
