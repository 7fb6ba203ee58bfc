"""GPU parity of the individual-particle path: scan, radix sort, cell offsets,
the reference's cell indices and the full binning step -- all bit-exact against
the oracle (stable sort / prefix sums / the CPU replay of the step)."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def _t(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).cuda()


def _np(t):
    return t.cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("n", [0, 1, 5, 4095, 4096, 4097, 8192, 16383, 16384, 16385, 2 * 16384 + 1, 100_003,
                               1 << 22, 1 << 26])
def test_exclusive_scan_bit_exact(gpgmp, n):
    from inchman_b200 import individual as ind
    rng = np.random.default_rng(n)
    x = rng.integers(0, 2**32, size=n, dtype=np.uint64).astype(np.uint32)
    if n:
        x[: min(n, 7)] = 0xFFFFFFFF   # wrap-around mod 2^32
    want = np.zeros(n, np.uint32)
    oracle.orc().orc_exclusive_scan_u32(oracle.ptr(x), oracle.ptr(want), n)
    if n == 0:
        return
    scratch = ind.scan_scratch(n)
    got = _np(ind.exclusive_scan_u32(_t(x), scratch))
    assert np.array_equal(got, want)
    assert ind.scratch_status(scratch, 0) == 0


@pytest.mark.parametrize("offset", [1, 2, 3])
def test_exclusive_scan_of_an_unaligned_view(gpgmp, offset):
    """Input that starts 4, 8 or 12 bytes past a 16-byte boundary (a slice of a larger
    buffer) is scanned element by element, with the same result; several 16384-value
    tiles take that path, so the look-back between them is crossed too."""
    from inchman_b200 import individual as ind
    n = 3 * 16384 + 17
    rng = np.random.default_rng(offset)
    x = rng.integers(0, 2**32, size=n + offset, dtype=np.uint64).astype(np.uint32)
    want = np.zeros(n, np.uint32)
    oracle.orc().orc_exclusive_scan_u32(oracle.ptr(np.ascontiguousarray(x[offset:])), oracle.ptr(want), n)
    view = _t(x)[offset:]
    assert view.data_ptr() % 16 != 0
    got = _np(ind.exclusive_scan_u32(view, ind.scan_scratch(n)))
    assert np.array_equal(got, want)


@pytest.mark.parametrize("n,bits", [(1, 32), (3839, 8), (3841, 20), (65536, 32), (1_000_003, 21), (1 << 22, 20),
                                    (7681, 10), (200_000, 16), (200_001, 17), (777_777, 26), (123_457, 30),
                                    (1 << 20, 24), (7680, 20), (2 * 7680 + 1, 20), (7680, 8), (3840, 8),
                                    (3841, 32), (2 * 3840 - 1, 16)])
def test_sort_pairs_stable_bit_exact(gpgmp, n, bits):
    from inchman_b200 import individual as ind
    rng = np.random.default_rng(bits + n)
    hi = 1 << bits
    keys = rng.integers(0, hi, size=n, dtype=np.uint64).astype(np.uint32)
    keys[::2] %= 4096          # many equal keys: stability matters
    vals = np.arange(n, dtype=np.uint32)
    wk, wv = keys.copy(), vals.copy()
    oracle.orc().orc_sort_pairs_u32(oracle.ptr(wk), oracle.ptr(wv), n)
    ko, vo, scratch = ind.sort_pairs_u32(_t(keys), _t(vals), bits)
    assert np.array_equal(_np(ko), wk)
    assert np.array_equal(_np(vo), wv)
    assert ind.scratch_status(scratch, 1, n, bits) == 0


@pytest.mark.parametrize("offset,n", [(1, 100_003), (2, 5), (3, 4 * 7680 + 3)])
def test_sort_of_unaligned_views(gpgmp, offset, n):
    """Keys and values that start 4, 8 or 12 bytes past a 16-byte boundary (views into
    larger buffers): the histogram's 16-byte loads start after the head, the result is
    the same stable sort."""
    from inchman_b200 import individual as ind
    rng = np.random.default_rng(offset)
    keys = rng.integers(0, 1 << 20, size=n + offset, dtype=np.uint64).astype(np.uint32)
    vals = np.arange(n + offset, dtype=np.uint32)
    wk, wv = keys[offset:].copy(), vals[offset:].copy()
    oracle.orc().orc_sort_pairs_u32(oracle.ptr(wk), oracle.ptr(wv), n)
    tk, tv = _t(keys)[offset:], _t(vals)[offset:]
    assert tk.data_ptr() % 16 != 0
    ko, vo, scratch = ind.sort_pairs_u32(tk, tv, 20)
    assert np.array_equal(_np(ko), wk) and np.array_equal(_np(vo), wv)
    assert ind.scratch_status(scratch, 1, n, 20) == 0


def test_sort_full_32_bit_keys_with_duplicates(gpgmp):
    from inchman_b200 import individual as ind
    rng = np.random.default_rng(11)
    n = 300_000
    keys = rng.integers(0, 2**32, size=n, dtype=np.uint64).astype(np.uint32)
    keys[n // 2:] = keys[: n - n // 2]          # many equal keys: stability matters
    vals = rng.integers(0, 2**32, size=n, dtype=np.uint64).astype(np.uint32)
    wk, wv = keys.copy(), vals.copy()
    oracle.orc().orc_sort_pairs_u32(oracle.ptr(wk), oracle.ptr(wv), n)
    ko, vo, _ = ind.sort_pairs_u32(_t(keys), _t(vals), 32)
    assert np.array_equal(_np(ko), wk) and np.array_equal(_np(vo), wv)


@pytest.mark.parametrize("ncells,n", [(16, 0), (16, 1), (1 << 10, 5000), (1 << 20, 1 << 22)])
def test_cell_offsets_and_reference_indices(gpgmp, ncells, n):
    from inchman_b200 import individual as ind
    rng = np.random.default_rng(ncells)
    keys = np.sort(rng.integers(0, ncells, size=n).astype(np.uint32))
    ws, wc = np.zeros(ncells, np.uint32), np.zeros(ncells, np.uint32)
    oracle.orc().orc_cell_offsets(oracle.ptr(keys), n, ncells, oracle.ptr(ws), oracle.ptr(wc))
    import torch
    tk = _t(keys) if n else torch.zeros(1, dtype=torch.int32, device="cuda")
    s, c = ind.cell_offsets(tk[:n] if n else tk[:0], ncells)
    assert np.array_equal(_np(s), ws) and np.array_equal(_np(c), wc)
    if n:
        wl, wr = np.zeros(ncells, np.uint32), np.zeros(ncells, np.uint32)
        oracle.orc().orc_cell_indices_ref(oracle.ptr(keys), n, ncells, oracle.ptr(wl), oracle.ptr(wr))
        left, right = ind.cell_indices(s, c)
        assert np.array_equal(_np(left), wl) and np.array_equal(_np(right), wr)


@pytest.mark.parametrize("n,grid,steps", [(10_000, 64, 5), (200_000, 256, 3), (1 << 22, 1024, 2)])
def test_particle_steps_bit_exact(gpgmp, n, grid, steps):
    from inchman_b200 import individual as ind
    x, y, sp = ind.uniform_particles(n, grid, seed=5)
    p = ind.Particles(n, grid, D=0.5, vx=0.1, vy=0.0, dt=1.0, p_react=0.05, seed=1234)
    p.set(x, y, sp, step=0)
    p.step(steps)
    gx, gy, gsp = p.get()
    assert p.status() == 0
    ox, oy, osp = x.copy(), y.copy(), sp.copy()
    m = oracle.orc().orc_particles_run(n, oracle.ptr(ox), oracle.ptr(oy), oracle.ptr(osp), grid, 0.5, 0.1, 0.0, 1.0,
                                       0.05, 1234, 0, steps)
    assert len(gx) == m
    assert np.array_equal(gx, ox[:m]) and np.array_equal(gy, oy[:m]) and np.array_equal(gsp, osp[:m])
    # removals come in A/B pairs
    assert (np.sum(gsp == 0) - np.sum(gsp == 1)) == (np.sum(sp == 0) - np.sum(sp == 1))
    assert m < n


@pytest.mark.gpu
@pytest.mark.parametrize("p_react", [0.05, 1.0])
def test_particle_steps_clustered_bit_exact(gpgmp, p_react):
    """Particles packed into 8 x 8 cells of a 128 x 128 grid: hundreds per cell, and
    more in one tile of cells than its shared-memory staging holds (the kernel then
    pairs and compacts those cells in global memory)."""
    from inchman_b200 import individual as ind
    n, grid, steps = 30_000, 128, 3
    rng = np.random.default_rng(17)
    x = rng.uniform(60.0, 68.0, n).astype(np.float32)
    y = rng.uniform(60.0, 68.0, n).astype(np.float32)
    sp = rng.integers(0, 2, n).astype(np.uint8)
    p = ind.Particles(n, grid, D=0.05, vx=0.0, vy=0.0, dt=1.0, p_react=p_react, seed=99)
    p.set(x, y, sp, step=0)
    p.step(steps)
    gx, gy, gsp = p.get()
    assert p.status() == 0
    ox, oy, osp = x.copy(), y.copy(), sp.copy()
    m = oracle.orc().orc_particles_run(n, oracle.ptr(ox), oracle.ptr(oy), oracle.ptr(osp), grid, 0.05, 0.0, 0.0, 1.0,
                                       p_react, 99, 0, steps)
    assert len(gx) == m and m < n
    assert np.array_equal(gx, ox[:m]) and np.array_equal(gy, oy[:m]) and np.array_equal(gsp, osp[:m])


@pytest.mark.parametrize("clustered", [False, True])
def test_particle_bins_follow_the_step(gpgmp, clustered):
    """Without reactions a step keeps every particle, in cell order: the bins of the
    step (start, count, sorted keys) are those of the positions it returns."""
    from inchman_b200 import individual as ind
    n, grid = 50_000, 128
    if clustered:
        rng = np.random.default_rng(3)
        x = rng.uniform(30.0, 34.0, n).astype(np.float32)
        y = rng.uniform(90.0, 92.0, n).astype(np.float32)
        sp = rng.integers(0, 2, n).astype(np.uint8)
    else:
        x, y, sp = ind.uniform_particles(n, grid, seed=8)
    p = ind.Particles(n, grid, D=0.3, vx=0.2, vy=-0.1, dt=1.0, p_react=0.0, seed=4)
    p.set(x, y, sp, step=0)
    p.step(1)
    gx, gy, gsp = p.get()
    start, count, keys, idx = p.bins()
    cells = gy.astype(np.int64) * grid + gx.astype(np.int64)
    assert len(gx) == n and np.all(np.diff(cells) >= 0)
    want = np.bincount(cells, minlength=grid * grid)
    assert np.array_equal(count, want)
    assert np.array_equal(start, (np.cumsum(want) - want).astype(np.uint32))
    assert np.array_equal(keys, cells.astype(np.uint32))
    assert np.array_equal(np.sort(idx), np.arange(n, dtype=np.uint32))


@pytest.mark.parametrize("case", ["empty", "single", "all_a", "no_reaction", "full_reaction"])
def test_particle_step_edge_cases(gpgmp, case):
    """Edge cases of the particle step against the oracle: no particles, one particle,
    one species only (no pairs), p = 0 (everyone stays) and p = 1."""
    from inchman_b200 import individual as ind
    grid, steps = 64, 3
    n = {"empty": 0, "single": 1}.get(case, 5000)
    rng = np.random.default_rng(23)
    x = rng.uniform(0.0, grid, n).astype(np.float32)
    y = rng.uniform(0.0, grid, n).astype(np.float32)
    sp = (np.zeros(n) if case == "all_a" else rng.integers(0, 2, n)).astype(np.uint8)
    p_react = {"no_reaction": 0.0, "full_reaction": 1.0}.get(case, 0.3)
    p = ind.Particles(max(n, 1), grid, D=0.4, vx=0.05, vy=0.02, dt=1.0, p_react=p_react, seed=7)
    p.set(x, y, sp, step=0)
    p.step(steps)
    gx, gy, gsp = p.get()
    assert p.status() == 0
    ox, oy, osp = x.copy(), y.copy(), sp.copy()
    m = oracle.orc().orc_particles_run(n, oracle.ptr(ox), oracle.ptr(oy), oracle.ptr(osp), grid, 0.4, 0.05, 0.02,
                                       1.0, p_react, 7, 0, steps) if n else 0
    assert len(gx) == m
    assert np.array_equal(gx, ox[:m]) and np.array_equal(gy, oy[:m]) and np.array_equal(gsp, osp[:m])
    if case in ("all_a", "no_reaction"):
        assert m == n
    # the last step's bins hold the particles it started with
    start, count, _, _ = p.bins()
    assert int(count.sum()) >= len(gx)
    if case in ("all_a", "no_reaction", "empty", "single"):
        assert int(count.sum()) == len(gx)
    assert np.array_equal(start, (np.cumsum(count) - count).astype(np.uint32))


@pytest.mark.parametrize("bits", [20, 32])
def test_sort_at_2p28_pairs_size_independent_properties(gpgmp, bits):
    """2^28 pairs (about 7 GB on the device, 70,000 tiles, counts far above 16 bits in
    the look-back words): too large for the oracle, so the size-independent properties
    of a stable sort, checked on the device -- keys in order, equal keys in input order
    (the values are the input indices), every output pair taken from its input index,
    and the values a permutation."""
    import torch
    from inchman_b200 import individual as ind
    n = 1 << 28
    g = torch.Generator(device="cuda").manual_seed(bits)
    keys = torch.randint(0, 1 << 31, (n,), dtype=torch.int64, device="cuda", generator=g)
    if bits < 32:
        keys &= (1 << bits) - 1
    else:
        keys = keys * 2 + (keys & 1)      # use the top bit too
    keys = keys.to(torch.uint32).view(torch.int32) if hasattr(torch, "uint32") else keys.to(torch.int32)
    vals = torch.arange(n, dtype=torch.int32, device="cuda")
    ko, vo, scratch = ind.sort_pairs_u32(keys, vals, bits)
    torch.cuda.synchronize()
    assert ind.scratch_status(scratch, 1, n, bits) == 0
    k64 = ko.to(torch.int64) & 0xFFFFFFFF
    assert bool((k64[1:] >= k64[:-1]).all())
    same = k64[1:] == k64[:-1]
    assert bool((vo[1:][same] > vo[:-1][same]).all())
    assert torch.equal(ko, keys[vo.long()])
    seen = torch.zeros(n, dtype=torch.int32, device="cuda")
    seen.index_put_((vo.long(),), torch.ones(n, dtype=torch.int32, device="cuda"), accumulate=True)
    assert bool((seen == 1).all())


def test_scan_at_2p29_values_size_independent_properties(gpgmp):
    """2^29 values (4 GB in and out, 32,768 tiles, sums that wrap modulo 2^32): the
    defining property of the exclusive scan checked on the device, in chunks --
    out[0] = 0 and out[i + 1] - out[i] = in[i] modulo 2^32 -- and no look-back timeout."""
    import torch
    from inchman_b200 import individual as ind
    n = 1 << 29
    g = torch.Generator(device="cuda").manual_seed(29)
    x = torch.randint(-(1 << 31), 1 << 31, (n,), dtype=torch.int64, device="cuda", generator=g).to(torch.int32)
    scratch = ind.scan_scratch(n)
    out = ind.exclusive_scan_u32(x, scratch)
    torch.cuda.synchronize()
    assert ind.scratch_status(scratch, 0, n) == 0
    assert int(out[0]) == 0
    step = 1 << 26
    for a in range(0, n - 1, step):
        b = min(a + step, n - 1)
        d = (out[a + 1:b + 1].to(torch.int64) - out[a:b].to(torch.int64)) & 0xFFFFFFFF
        assert torch.equal(d, x[a:b].to(torch.int64) & 0xFFFFFFFF), a
