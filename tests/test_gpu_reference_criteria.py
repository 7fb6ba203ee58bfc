"""The reference's own validation criteria (python/gpgmp/test/*.py) run against the
GPU solvers, with the models of the reference's example files, and the statistical
agreement of the GPU solver with the reference-exact restatement over 10^4
realisations."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def test_ab_reaction_means(gpgmp):
    """doc/examples/ABReaction.xml: 256 x 256, L = 40, no diffusion, 2A->0 (1e-3,
    hazard k A (A-1)), A+B->0 (1e-2), 0->A (1.2), 0->B (1.0), t = 1000, outputs
    every 10.  Pass: final <A> = 9.6 and <B> = 12.1 within 1 %
    (python/gpgmp/test/abreaction.py:111-118)."""
    from inchman_b200.model import DiffusionModel
    from inchman_b200.solver import Solver
    m = DiffusionModel(width=256, height=256, physical_length=40.0, p0=0.1, max_time=1000.0, output_interval=10.0)
    m.add_species("A", 0.0).add_species("B", 0.0)
    m.add_reaction("AAAnnihilation", {"A": 2}, {}, 1e-3)
    m.add_reaction("ABAnnihilation", {"A": 1, "B": 1}, {}, 1e-2)
    m.add_reaction("ACreation", {}, {"A": 1}, 1.2)
    m.add_reaction("BCreation", {}, {"B": 1}, 1.0)
    with Solver(m, realisations=1, seed=2012) as s:
        snaps, times, steps = s.solve(max_snapshots=2)   # initial and first output only
        final = s.get_state()[0]
    a, b = final[0].mean(), final[1].mean()
    assert abs(a - 9.6) / 9.6 <= 0.01, a
    assert abs(b - 12.1) / 12.1 <= 0.01, b


def test_homogeneous_point_source_diffusion(gpgmp):
    """doc/examples/HomogeneousDiffusion.xml: 128 x 128, L = 100, D = 1, 1e5
    molecules in cell (64, 64), t = 40.  Pass: RMSE of the x and y slices through
    the centre against the 2-D Gaussian <= 5e-4
    (python/gpgmp/test/homogeneous_diffusion.py:16-22, 74-82)."""
    from inchman_b200.model import Compartment, DiffusionModel
    from inchman_b200.solver import Solver
    nx, L, D, N, T = 128, 100.0, 1.0, 1e5, 40.0
    m = DiffusionModel(width=nx, height=nx, physical_length=L, p0=0.1, max_time=T, output_interval=1.0)
    m.add_species("A", D)
    init = np.zeros((1, 1, nx, nx), np.int32)
    init[0, 0, 64, 64] = int(N)
    with Solver(m, realisations=1, seed=77) as s:
        s.set_state(init)
        snaps, times, steps = s.solve(max_snapshots=64)
    t = float(times[-1])
    nav = snaps[-1, 0, 0].astype(np.float64)
    dx = L / nx
    xg = np.arange(nx) * dx - L / 2.0

    def gauss(x, y):
        return 1.0 / (4.0 * D * np.pi * t) * np.exp(-(x * x + y * y) / (4.0 * D * t))

    rmsex = np.sqrt(np.sum((nav[nx // 2, :] / (N * dx * dx) - gauss(xg, xg[nx // 2])) ** 2) / nx)
    rmsey = np.sqrt(np.sum((nav[:, nx // 2] / (N * dx * dx) - gauss(xg, xg[nx // 2])) ** 2) / nx)
    assert nav.sum() == N                       # reflecting walls conserve particles
    assert rmsex <= 5e-4 and rmsey <= 5e-4, (rmsex, rmsey)


def test_statistics_match_reference_exact_restatement_1e4_realisations(gpgmp):
    """A+B <-> C with diffusion on an 8 x 8 lattice (one absorbing wall), t = 0.2,
    10,000 realisations from one initial state: per-cell, per-species mean (z-test),
    variance (F-test) and distribution (two-sample KS) of the GPU solver against the
    reference-exact restatement (Threefry keyed per cell, one uniform per particle,
    the reference's seeding pattern), Bonferroni-corrected alpha = 1e-3."""
    from scipy import stats
    from helpers import small_homog
    from inchman_b200.solver import Solver
    m = small_homog(W=8, H=8, max_time=0.2, bmask=(0, 1, 0, 0))
    for sp, lam in zip(m.species, (20.0, 15.0, 3.0)):
        sp.initial = lam
    desc, keep = m.to_desc()
    R = 10_000
    init = oracle.init_poisson(m.width, m.height, m.num_species, 1, 5, [s.initial for s in m.species])
    with Solver(m, realisations=R, seed=4242) as s:
        s.set_state(np.repeat(init, R, axis=0))
        s.solve(count_only=True)
        gpu = s.get_state().reshape(R, -1).astype(np.float64)
    ref = np.zeros((R,) + init.shape[1:], np.int32)
    oracle.orc().orc_ref_solve_many(oracle.model_ptr(desc), oracle.ptr(init), R, 1000, oracle.ptr(ref))
    ref = ref.reshape(R, -1).astype(np.float64)
    k = gpu.shape[1]
    alpha = 1e-3 / (3 * k)
    se = np.sqrt(gpu.var(0, ddof=1) / R + ref.var(0, ddof=1) / R) + 1e-12
    z = np.abs(gpu.mean(0) - ref.mean(0)) / se
    assert (z < stats.norm.isf(alpha / 2)).all(), z.max()
    vg, vr = gpu.var(0, ddof=1), ref.var(0, ddof=1)
    ok = (vr == 0) & (vg == 0)
    f = vg / np.where(vr > 0, vr, 1)
    lo, hi = stats.f.ppf(alpha / 2, R - 1, R - 1), stats.f.isf(alpha / 2, R - 1, R - 1)
    assert (ok | ((f > lo) & (f < hi))).all()
    pmin = min(stats.ks_2samp(gpu[:, j], ref[:, j]).pvalue for j in range(k))
    assert pmin > alpha, pmin


def test_homogeneous_drift_diffusion(gpgmp):
    """doc/examples/HomogeneousDrift.xml: inhomogeneous solver, 512 x 512, L = 32,
    Dx = 0.6, Dy = 0.8, drift (0.8, 0.4), 1e5 molecules in cell (256, 256), t = 5,
    10 runs.  Pass: RMSE of the mean final density against the drifted 2-D Gaussian
    <= 1e-4 (python/gpgmp/test/homogeneous_drift_diffusion.py:27, 117, 140).  The
    drift moves the centre by (4, 2); the test also checks that mean position."""
    from inchman_b200 import _lib
    from inchman_b200.model import DiffusionModel
    from inchman_b200.solver import Solver
    nx, L, N, T, runs = 512, 32.0, 100_000, 5.0, 10
    m = DiffusionModel(width=nx, height=nx, physical_length=L, p0=0.1, max_time=T, output_interval=1.0,
                       solver=_lib.STOCHASTIC_INHOMOGENEOUS, drift_method=_lib.DRIFT_HOMOGENEOUS,
                       drift_params=(0.6, 0.8, 0.8, 0.4, 0, 0, 0, 0))
    m.add_species("A", 1.0)
    init = np.zeros((runs, 1, nx, nx), np.int32)
    init[:, 0, 256, 256] = N
    with Solver(m, realisations=runs, seed=3) as s:
        s.set_state(init)
        snaps, times, steps = s.solve(max_snapshots=8)
    sample_t = float(times[-1])                 # the last output, as the reference samples it
    final = snaps[-1][:, 0].astype(np.float64)
    dx = L / nx
    xc = np.arange(nx) * dx - L / 2.0
    nstate = final.mean(axis=0)

    def biased(xc, yc, t, dxc, dyc, qx, qy):
        gx = np.outer(xc, np.ones_like(xc))
        gy = np.outer(np.ones_like(yc), yc)
        px = 1.0 / np.sqrt(4.0 * dxc * np.pi * t) * np.exp(-((gx - t * qx) ** 2) / (4.0 * dxc * t))
        py = 1.0 / np.sqrt(4.0 * dyc * np.pi * t) * np.exp(-((gy - t * qy) ** 2) / (4.0 * dyc * t))
        return px * py

    # first array axis is y (D = 0.8, drift 0.4), second is x (D = 0.6, drift 0.8),
    # the argument order of the reference's call
    theo = biased(xc, xc, sample_t, 0.8, 0.6, 0.4, 0.8) * dx * dx
    rmse = np.sqrt(np.sum((nstate / nstate.sum() - theo) ** 2) / nx / nx)
    assert rmse <= 1e-4, rmse
    w = nstate / nstate.sum()
    mx = (w.sum(axis=0) * xc).sum()
    my = (w.sum(axis=1) * xc).sum()
    assert abs(mx - 0.8 * sample_t) < 0.05 and abs(my - 0.4 * sample_t) < 0.05, (mx, my)
    assert (nstate.sum() == N) and sample_t >= T - 1.0
