"""Individual-particle population bookkeeping (IndividualSolver::maintainPopulation,
IndividualSolver.cpp:458-671): the oracle's restatement against invariants and
uniformity on the CPU, and the CUDA path bit for bit against the oracle."""
import ctypes as C

import numpy as np
import pytest

import oracle


def _case(rng, ncells, mean, capacity_extra, change):
    counts = rng.poisson(mean, ncells).astype(np.uint32)
    n = int(counts.sum())
    keys = np.repeat(np.arange(ncells, dtype=np.uint32), counts)
    ids = rng.permutation(n + capacity_extra).astype(np.uint32)
    active, pool = ids[:n].copy(), ids[n:].copy()
    start = np.concatenate([[0], np.cumsum(counts)[:-1]]).astype(np.uint32)
    goal = np.maximum(counts.astype(np.int64) + rng.integers(-change, change + 1, ncells), 0).astype(np.int32)
    return keys, active, start, counts, goal, pool


def _oracle(keys, ids, start, count, goal, pool, seed, step):
    n, npool = len(keys), len(pool)
    cap = n + npool + 1
    ko = np.zeros(cap, np.uint32); io = np.zeros(cap, np.uint32); po = np.zeros(cap, np.uint32)
    na, npo = C.c_int64(0), C.c_int64(0)
    rc = oracle.orc().orc_population_maintain(oracle.ptr(keys), oracle.ptr(ids), n, oracle.ptr(start),
                                              oracle.ptr(count), oracle.ptr(goal), len(goal), oracle.ptr(pool),
                                              npool, seed, step, oracle.ptr(ko), oracle.ptr(io), oracle.ptr(po),
                                              C.byref(na), C.byref(npo))
    return rc, ko[:na.value], io[:na.value], po[:npo.value]


def test_oracle_invariants():
    rng = np.random.default_rng(1)
    keys, ids, start, count, goal, pool = _case(rng, 500, 4.0, 3000, 3)
    rc, ko, io, po = _oracle(keys, ids, start, count, goal, pool, 7, 3)
    assert rc == 0
    assert np.array_equal(np.bincount(ko, minlength=500), goal)           # counts reached
    assert np.all(np.diff(ko.astype(np.int64)) >= 0)                      # still sorted by cell
    assert len(np.unique(np.concatenate([io, po]))) == len(ids) + len(pool)   # no id lost or doubled
    for c in np.flatnonzero(goal < count)[:50]:                           # removals come from the cell
        old = set(ids[start[c]:start[c] + count[c]].tolist())
        assert set(io[ko == c].tolist()) <= old


def test_oracle_removals_are_uniform():
    """Cell with 10 individuals, 3 removed: each is removed with probability 0.3."""
    n = 10
    keys = np.zeros(n, np.uint32); ids = np.arange(n, dtype=np.uint32)
    start = np.zeros(1, np.uint32); count = np.array([n], np.uint32); goal = np.array([7], np.int32)
    pool = np.arange(n, n + 5, dtype=np.uint32)
    hits = np.zeros(n)
    trials = 4000
    for step in range(trials):
        rc, ko, io, po = _oracle(keys, ids, start, count, goal, pool, 11, step)
        hits[po[:3]] += 1
    p = hits / trials
    assert np.all(np.abs(p - 0.3) < 4 * np.sqrt(0.3 * 0.7 / trials)), p


def test_oracle_reports_a_short_pool():
    keys = np.zeros(0, np.uint32)
    rc, *_ = _oracle(keys, keys, np.zeros(2, np.uint32), np.zeros(2, np.uint32), np.array([3, 2], np.int32),
                     np.arange(4, dtype=np.uint32), 1, 1)
    assert rc == -1


@pytest.mark.gpu
@pytest.mark.parametrize("ncells,mean,extra,change", [(1, 6.0, 10, 4), (97, 3.0, 400, 3), (4096, 0.5, 20000, 2),
                                                      (6145, 3.0, 20000, 3), (200_000, 5.0, 400_000, 2),
                                                      (50, 0.0, 100, 3)])
def test_gpu_matches_oracle(gpgmp, ncells, mean, extra, change):
    import torch
    from inchman_b200.individual import maintain_population
    rng = np.random.default_rng(ncells)
    keys, ids, start, count, goal, pool = _case(rng, ncells, mean, extra, change)
    for step in (0, 5):
        rc, ko, io, po = _oracle(keys, ids, start, count, goal, pool, 123, step)
        assert rc == 0
        t = lambda a, dt=torch.int32: torch.tensor(a.view(np.int32) if a.dtype == np.uint32 else a, dtype=dt,
                                                   device="cuda")
        gk, gi, gs, gp = maintain_population(t(keys), t(ids), t(start), t(count), t(goal), t(pool), 123, step)
        assert np.array_equal(gk.cpu().numpy().view(np.uint32), ko)
        assert np.array_equal(gi.cpu().numpy().view(np.uint32), io)
        assert np.array_equal(gp.cpu().numpy().view(np.uint32), po)
        want_start = np.concatenate([[0], np.cumsum(goal)[:-1]]).astype(np.uint32)
        assert np.array_equal(gs.cpu().numpy().view(np.uint32), want_start)


@pytest.mark.gpu
def test_gpu_reports_a_short_pool(gpgmp):
    import torch
    from inchman_b200 import _lib
    from inchman_b200.individual import maintain_population
    z = torch.zeros(0, dtype=torch.int32, device="cuda")
    with pytest.raises(_lib.GpgmpError):
        maintain_population(z, z, torch.zeros(2, dtype=torch.int32, device="cuda"),
                            torch.zeros(2, dtype=torch.int32, device="cuda"),
                            torch.tensor([3, 2], dtype=torch.int32, device="cuda"),
                            torch.arange(4, dtype=torch.int32, device="cuda"), 1, 1)


def _gpu_vs_oracle(keys, ids, start, count, goal, pool, seed, step):
    import torch
    from inchman_b200.individual import maintain_population
    rc, ko, io, po = _oracle(keys, ids, start, count, goal, pool, seed, step)
    assert rc == 0
    t = lambda a: torch.tensor(a.view(np.int32) if a.dtype == np.uint32 else a, dtype=torch.int32, device="cuda")
    gk, gi, gs, gp = maintain_population(t(keys), t(ids), t(start), t(count), t(goal), t(pool), seed, step)
    assert np.array_equal(gk.cpu().numpy().view(np.uint32), ko)
    assert np.array_equal(gi.cpu().numpy().view(np.uint32), io)
    assert np.array_equal(gp.cpu().numpy().view(np.uint32), po)


@pytest.mark.gpu
def test_gpu_heavy_cells(gpgmp):
    """One cell loses 15,000 of 20,000 individuals, another gains 29,997; the rest
    are ordinary: the per-cell loops and the individual-parallel moves agree with
    the oracle bit for bit."""
    rng = np.random.default_rng(7)
    ncells = 3000
    counts = rng.poisson(2.0, ncells).astype(np.uint32)
    counts[17] = 20000
    counts[2500] = 3
    n = int(counts.sum())
    keys = np.repeat(np.arange(ncells, dtype=np.uint32), counts)
    allids = rng.permutation(n + 40000).astype(np.uint32)
    ids, pool = allids[:n].copy(), allids[n:].copy()
    start = np.concatenate([[0], np.cumsum(counts)[:-1]]).astype(np.uint32)
    goal = np.maximum(counts.astype(np.int64) + rng.integers(-2, 3, ncells), 0).astype(np.int32)
    goal[17] = 5000
    goal[2500] = 30000
    goal[5] = -4                      # negative goals count as 0
    _gpu_vs_oracle(keys, ids, start, counts, goal, pool, 99, 2)


@pytest.mark.gpu
@pytest.mark.parametrize("which", ["list", "pool"])
def test_gpu_reports_full_outputs(gpgmp, which):
    import torch
    from inchman_b200 import _lib
    from inchman_b200.individual import maintain_population
    rng = np.random.default_rng(3)
    keys, ids, start, count, goal, pool = _case(rng, 500, 4.0, 3000, 3)
    t = lambda a: torch.tensor(a.view(np.int32) if a.dtype == np.uint32 else a, dtype=torch.int32, device="cuda")
    n_new = int(goal.sum())
    kw = {"capacity": n_new - 1} if which == "list" else {"pool_capacity": 10}
    with pytest.raises(_lib.GpgmpError):
        maintain_population(t(keys), t(ids), t(start), t(count), t(goal), t(pool), 1, 1, **kw)
    # exactly enough room succeeds
    gk, gi, gs, gp = maintain_population(t(keys), t(ids), t(start), t(count), t(goal), t(pool), 1, 1,
                                         capacity=n_new)
    assert gk.numel() == n_new
