"""The batched persistent ensemble kernel against the per-instance solvers (the
reference's one-solver-per-run structure) and against the oracle: bit-exact final
states, step counts, snapshots and status words."""
import numpy as np
import pytest

import oracle
from helpers import small_homog

pytestmark = pytest.mark.gpu


def test_replicated_model_matches_wide_solver_and_oracle(gpgmp):
    import torch
    from inchman_b200.ensemble import Ensemble, replicate
    from inchman_b200.solver import Solver
    m = small_homog(W=20, H=20, max_time=0.5, bmask=(0, 1, 0, 0))
    lam = [60.0, 40.0, 5.0]
    R, seed = 5, 321
    specs = replicate(m, lam, R, seed, max_snapshots=8)
    ens = Ensemble(specs)
    state = ens.alloc_state()
    snaps = ens.alloc_snapshots()
    ens.init_poisson(state)
    init = state.clone()
    ens.run(state, snaps)
    st, steps, times = ens.results()
    with Solver(m, realisations=R, seed=seed) as s:
        s.init_poisson(lam)
        ws, wt, wsteps = s.solve(max_snapshots=8)
        w_init = ws[0]
    got = np.stack([ens.instance_state(state, i).cpu().numpy() for i in range(R)])
    got_init = np.stack([ens.instance_state(init, i).cpu().numpy() for i in range(R)])
    assert np.array_equal(got_init, w_init)
    assert (steps == wsteps).all()
    assert np.array_equal(got, ws[-1])
    # snapshots: [instance][snapshot][S][H][W] vs [snapshot][R][S][H][W]
    S, H, W = ens.shapes[0]
    sn = snaps.cpu().numpy()
    k = len(wt)
    for i in range(R):
        o = ens.snap_offsets[i]
        mine = sn[o:o + k * S * H * W].reshape(k, S, H, W)
        assert np.array_equal(mine, ws[:, i])
        assert np.array_equal(times[i * 8:i * 8 + k], wt)
    desc, keep = m.to_desc()
    ost, osn, ot, osteps, _ = oracle.rep_solve(desc, w_init, R, seed, 8)
    assert np.array_equal(got, ost) and osteps == steps[0]


def test_random_heterogeneous_instances_match_their_own_solvers(gpgmp):
    import torch
    from inchman_b200.ensemble import Ensemble, random_ensemble
    from inchman_b200.solver import Solver
    specs = random_ensemble(12, seed=99, max_time=0.3)
    ens = Ensemble(specs)
    for thr, cps in [(256, 4), (128, 8), (512, 1)]:
        ens.configure(thr, cps)
        state = ens.alloc_state()
        ens.init_poisson(state)
        ens.run(state)
        st, steps, _ = ens.results()
        for i, sp in enumerate(specs):
            with Solver(sp.model, realisations=1, seed=sp.seed, sync_each_launch=True) as s:
                s.init_poisson(sp.lam)
                snaps, times, n = s.solve(max_snapshots=4)
                assert n == steps[i], (i, n, steps[i])
                assert np.array_equal(ens.instance_state(state, i).cpu().numpy(), snaps[-1][0]), i
                assert s.status()[0] == st[i]


def test_graph_replay_reproduces(gpgmp):
    from inchman_b200.ensemble import Ensemble, random_ensemble
    specs = random_ensemble(40, seed=5, max_time=0.2)
    ens = Ensemble(specs)
    state = ens.alloc_state()
    ens.init_poisson(state)
    ens.run(state)
    a = state.clone()
    ens.init_poisson(state)
    ens.run(state)             # replay of the captured graph
    assert bool((a == state).all())
