"""GPU parity of the multi-cluster float32 Gray-Scott forward kernel.

The multi-cluster kernel spreads one 256 x 256 lattice over 2, 4 or 8 thread-block
clusters with G ghost rows per band side, swapped through global memory every G
steps.  Each band row sees exactly the values of the single-cluster kernel, so every
configuration must give the same bits: final state and every stored checkpoint, at
step counts around the swap period (G - 1, G, G + 1, 2G + 1), with and without drift,
and bit for bit against the oracle's float32 restatement over 1000 steps."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def _variants():
    from inchman_b200.gray_scott import MULTI_CLUSTER
    return sorted(MULTI_CLUSTER)


def _cfg(**kw):
    from inchman_b200.gray_scott import GrayScottConfig
    return GrayScottConfig(**kw)


def _run(cfg, variant, tu, tv, every, steps):
    import torch
    from inchman_b200 import gray_scott as gs
    n = cfg.n
    nck = max(1, -(-steps // every))
    ck = torch.full((nck, 2, n, n), float("nan"), device="cuda")
    u, v = gs.forward(tu, tv, cfg.params(variant=variant, checkpoint_every=every), checkpoints=ck if steps else None)
    torch.cuda.synchronize()
    return u, v, ck


def _fits(variant):
    """Whether the device holds all clusters of the variant at once (else the library
    refuses the launch with an error; it never starts a kernel that could wait on a
    cluster that is not running)."""
    import torch
    from inchman_b200 import _lib
    cfg = _cfg(n=256, steps=1)
    t = torch.zeros((256, 256), device="cuda")
    try:
        _run(cfg, variant, t, t, 1, 1)
    except _lib.GpgmpError:
        return False
    return True


@pytest.mark.parametrize("steps,drift,every", [(0, False, 1), (1, True, 1), (7, False, 3), (8, True, 8),
                                               (9, False, 2), (16, True, 5), (17, False, 1), (33, True, 4),
                                               (31, False, 3), (32, True, 1), (65, False, 9), (301, True, 7), (1000, False, 100)])
def test_multicluster_forward_bit_identical_to_single_cluster(gpgmp, steps, drift, every):
    import torch
    from inchman_b200 import gray_scott as gs
    cfg = _cfg(n=256, steps=steps, vx=0.05 if drift else 0.0, vy=-0.03 if drift else 0.0)
    u0, v0 = cfg.initial_state(np.float32)
    tu, tv = torch.tensor(u0, device="cuda"), torch.tensor(v0, device="cuda")
    ru, rv, rck = _run(cfg, 3, tu, tv, every, steps)
    ran = 0
    for var in _variants():
        if not _fits(var):
            continue
        u, v, ck = _run(cfg, var, tu, tv, every, steps)
        assert torch.equal(u, ru) and torch.equal(v, rv), (var, int((u != ru).sum()), int((v != rv).sum()))
        if steps:
            assert torch.equal(ck, rck), var
        ran += 1
    assert ran >= 1, "no multi-cluster configuration fits this device"
    assert gs.status() == 0


def test_multicluster_forward_bit_exact_against_oracle(gpgmp):
    """The automatic 4-cluster configuration (8 ghost rows), 1000 steps with drift, bit
    for bit against the oracle's float32 restatement of the kernels' operation order."""
    import torch
    from inchman_b200 import gray_scott as gs
    cfg = _cfg(n=256, steps=1000, vx=0.05, vy=-0.03, variant=41)
    if not _fits(41):
        pytest.skip("4 clusters of 16 CTAs are not co-resident on this device")
    u0, v0 = cfg.initial_state(np.float32)
    tu, tv = torch.tensor(u0, device="cuda"), torch.tensor(v0, device="cuda")
    u, v = gs.forward(tu, tv, cfg.params())
    torch.cuda.synchronize()
    gu, gv = u.cpu().numpy(), v.cpu().numpy()
    ou, ov = u0.astype(np.float32).copy(), v0.astype(np.float32).copy()
    oracle.orc().orc_gs_forward_f32(cfg.n, cfg.steps, cfg.F, cfg.k, cfg.Du, cfg.Dv, cfg.vx, cfg.vy, cfg.dt,
                                    oracle.ptr(ou), oracle.ptr(ov))
    assert gs.status() == 0
    assert np.array_equal(gu.view(np.uint32), ou.view(np.uint32)), int((gu != ou).sum())
    assert np.array_equal(gv.view(np.uint32), ov.view(np.uint32)), int((gv != ov).sum())


def test_automatic_choice_is_the_multicluster_kernel(gpgmp):
    """On a B200 variant 0 resolves to four clusters for 256 x 256 (the device holds
    them at once) and runs it: same bits as naming variant 41, with and without drift."""
    import torch
    from inchman_b200 import gray_scott as gs
    for drift in (False, True):
        assert gs.auto_variant(256, drift) == 41
        cfg = _cfg(n=256, steps=50, vx=0.05 if drift else 0.0, vy=-0.03 if drift else 0.0)
        u0, v0 = cfg.initial_state(np.float32)
        tu, tv = torch.tensor(u0, device="cuda"), torch.tensor(v0, device="cuda")
        a = _run(cfg, 0, tu, tv, 7, 50)
        b = _run(cfg, 41, tu, tv, 7, 50)
        assert all(torch.equal(x, y) for x, y in zip(a, b))
    assert gs.auto_variant(128) == 14   # one cluster, 4 warps per CTA
    assert gs.status() == 0


@pytest.mark.parametrize("steps,drift,every", [(1, False, 100), (17, True, 5), (250, False, 100), (301, True, 40)])
def test_multicluster_adjoint_matches_single_cluster(gpgmp, steps, drift, every):
    """The multi-cluster adjoint (with the multi-cluster recomputation of the segments)
    gives the same bits of lambda at the initial state as the single-cluster adjoint,
    and the same parameter gradient up to the order of its float partial sums (one row
    per lane instead of two): within 1e-4 of the largest component, far below the
    float32 gradient's own error against float64 and far above what a ghost row counted
    or a band row dropped would leave (about 1/256 of a component)."""
    import torch
    from inchman_b200 import gray_scott as gs
    cfg = _cfg(n=256, steps=steps, vx=0.05 if drift else 0.0, vy=-0.03 if drift else 0.0, checkpoint_every=every)
    u0, v0 = cfg.initial_state(np.float32)
    tu, tv = torch.tensor(u0, device="cuda"), torch.tensor(v0, device="cuda")
    g = torch.Generator(device="cuda").manual_seed(steps)
    lu = torch.rand((256, 256), device="cuda", generator=g) - 0.5
    lv = torch.rand((256, 256), device="cuda", generator=g) - 0.5

    def grad(variant):
        p = cfg.params(variant=variant)
        nck = -(-steps // every)
        ck = torch.empty((nck, 2, 256, 256), device="cuda")
        gs.forward(tu, tv, p, checkpoints=ck)
        out = gs.adjoint(p, ck, lu, lv)
        torch.cuda.synchronize()
        return out

    ru, rv, rg = grad(3)
    ran = 0
    for var in [0] + _variants():   # 0: single-cluster recomputation beside the multi-cluster adjoint
        if var and not _fits(var):
            continue
        mu, mv, mg = grad(var)
        assert torch.equal(mu, ru) and torch.equal(mv, rv), (var, int((mu != ru).sum()), int((mv != rv).sum()))
        scale = float(rg.abs().max())
        assert float((mg - rg).abs().max()) <= 1e-4 * scale, (var, (mg - rg).tolist(), rg.tolist())
        ran += 1
    assert ran >= 1
    assert gs.status() == 0


def test_multicluster_forwards_on_two_streams_and_in_a_graph(gpgmp):
    """Each multi-cluster launch takes its own exchange buffer from the stream-ordered
    pool and clears it on its stream: two solves on two streams at once, and two
    replays of a captured graph, give the bits of a solve on its own."""
    import torch
    from inchman_b200 import gray_scott as gs
    cfg = _cfg(n=256, steps=200, vx=0.05, vy=-0.03)
    if not _fits(41):
        pytest.skip("4 clusters of 16 CTAs are not co-resident on this device")
    p = cfg.params(variant=41)
    u0, v0 = cfg.initial_state(np.float32)
    tu, tv = torch.tensor(u0, device="cuda"), torch.tensor(v0, device="cuda")
    ru, rv = gs.forward(tu, tv, p)
    torch.cuda.synchronize()
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()
    with torch.cuda.stream(s1):
        a = gs.forward(tu, tv, p)
    with torch.cuda.stream(s2):
        b = gs.forward(tu, tv, p)
    torch.cuda.synchronize()
    for u, v in (a, b):
        assert torch.equal(u, ru) and torch.equal(v, rv)
    # graph capture: the launch, its pool allocation and the buffer clear are replayed
    s3 = torch.cuda.Stream()
    s3.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s3):
        gs.forward(tu, tv, p)              # warm up on the capturing stream
    torch.cuda.current_stream().wait_stream(s3)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        gu, gv = gs.forward(tu, tv, p)
    for _ in range(2):
        g.replay()
        torch.cuda.synchronize()
        assert torch.equal(gu, ru) and torch.equal(gv, rv)
    del g
    assert gs.status() == 0
