"""Launch shapes of the stochastic kernels and their autotuner: every diffusion tile
shape and SSA block size gives the same bits (the draws are keyed by cell, not by
thread), and gpgmp_solver_autotune leaves the state, clocks and status as they were."""
import numpy as np
import pytest

import oracle
from helpers import small_homog, small_inhom

pytestmark = pytest.mark.gpu


def _run(m, init, R, seed, tile=None, ssa=None, tune=False):
    from inchman_b200.solver import Solver
    with Solver(m, realisations=R, seed=seed) as s:
        s.set_state(init)
        if tile is not None:
            s.set_launch(tile, ssa)
        if tune:
            before = s.get_state()
            d = s.autotune(reps=2, cache=False)
            assert np.array_equal(s.get_state(), before)
            assert (s.status() == 0).all()
            assert set(d["ms_tiles"]) and all(v > 0 for v in d["ms_tiles"].values())
        snaps, times, steps = s.solve(max_snapshots=8)
        return snaps, times, steps, s.get_launch()


@pytest.mark.parametrize("kind", ["homogeneous", "inhomogeneous", "masked"])
def test_every_launch_shape_gives_the_same_bits(gpgmp, kind):
    from inchman_b200.solver import Solver
    if kind == "inhomogeneous":
        m = small_inhom(W=37, H=29, max_time=0.2)
        lam = [50.0, 50.0]
    else:
        m = small_homog(W=45, H=23, max_time=0.3, bmask=(0, 1, 0, 1))
        lam = [60.0, 40.0, 5.0]
        if kind == "masked":
            m.reactions[0].regions = [(0, 0, 20, 22)]
    R, seed = 3, 321
    init = oracle.init_poisson(m.width, m.height, m.num_species, R, 2, lam)
    base = _run(m, init, R, seed)
    assert base[3] == ((32, 16), 128)
    tiles, ssas = Solver.launch_choices()
    assert len(tiles) >= 4 and len(ssas) >= 2
    for k, tile in enumerate(tiles):
        ssa = ssas[k % len(ssas)]
        got = _run(m, init, R, seed, tile, ssa)
        assert got[3] == (tuple(tile), ssa)
        assert got[2] == base[2] and np.array_equal(got[1], base[1])
        assert np.array_equal(got[0], base[0]), (tile, ssa)
    tuned = _run(m, init, R, seed, tune=True)
    assert np.array_equal(tuned[0], base[0]) and tuned[2] == base[2]


def test_launch_shape_outside_the_choices_is_rejected(gpgmp):
    from inchman_b200 import _lib
    from inchman_b200.solver import Solver
    m = small_homog(W=8, H=8)
    with Solver(m, realisations=1, seed=1) as s:
        with pytest.raises(_lib.GpgmpError):
            s.set_launch((24, 24), 128)
        with pytest.raises(_lib.GpgmpError):
            s.set_launch((32, 16), 96)
        assert s.get_launch() == ((32, 16), 128)
