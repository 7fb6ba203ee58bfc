"""Benchmark workloads besides the default Gray-Scott line (bench.py --workload ...).

Each returns one JSON-ready dict in bench.py's format.  Inputs are synthetic and
seeded.  Units:
  cell-steps/s      lattice cells x realisations x event-loop steps per second
  particle-steps/s  particles x steps per second
  individuals/s     individuals in the list x bookkeeping calls per second
  individual-sweeps/s  individuals x directional sweeps per second
"""
from __future__ import annotations

import time

import numpy as np

METRIC = "cell-steps/s per B200, batched vs plain at same stats; adjoint/forward time ratio"


def _events():
    import torch
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def _base(args, world, metric_value, unit, workload, cfg, ms_per_step, extra):
    d = {"metric": METRIC, "value": metric_value, "unit": unit, "n_gpus": world, "steps": args.steps,
         "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
         "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded)",
         "config": dict({"workload": workload}, **cfg)}
    d.update(extra)
    return d


def ssa_plain(args, rank, world):
    """Homogeneous SSA + diffusion, 32 x 32, A+B<->C, 16 realisations, t = 10:
    the reference's structure (one solver per realisation, a wait after every launch)
    against the persistent batched kernel and the wide solver (one launch per kernel
    for all 16 realisations).  Plain realisation r and batched instance r use the same
    random streams (key (seed + r, 0)), so their final states are bit-identical: the
    same statistics by construction; the wide solver keys realisation r as (seed, r)."""
    import torch
    from .model import plain_ssa_model
    from .solver import Solver
    m = plain_ssa_model(width=32, max_time=10.0)
    R, seed = 16, 1234
    lam = [100.0, 100.0, 0.0]
    finals = {}

    def run_plain():
        steps, out = 0, []
        for r in range(R):
            with Solver(m, realisations=1, seed=seed + r, sync_each_launch=True) as s:
                s.init_poisson(lam)
                _, _, n = s.solve(count_only=True)
                out.append(s.get_state()[0])
                steps += n
        finals["plain"] = np.stack(out)
        return steps

    def run_wide():
        with Solver(m, realisations=R, seed=seed) as s:
            s.init_poisson(lam)
            _, _, n = s.solve(count_only=True)
        return n * R

    from .ensemble import Ensemble, InstanceSpec, autotune
    specs = [InstanceSpec(m, list(lam), seed + r, 0) for r in range(R)]
    (thr, cps), _ = autotune(specs)
    ens = Ensemble(specs)
    ens.configure(thr, cps)
    est = ens.alloc_state()

    def run_batched():
        ens.init_poisson(est)
        ens.run(est)
        _, st, _ = ens.results()
        finals["batched"] = est.view(R, m.num_species, m.height, m.width).cpu().numpy()
        return int(st.sum())

    res = {}
    for name, fn in (("plain", run_plain), ("wide", run_wide), ("batched", run_batched)):
        fn()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        steps = fn()
        torch.cuda.synchronize()
        t = time.perf_counter() - t0
        res[name] = (m.area * steps / t, t)
    same = bool(np.array_equal(finals["plain"], finals["batched"]))
    return _base(args, world, res["batched"][0], "cell-steps/s", "ssa_homogeneous_32x32_ABC_16real_t10",
                 {"grid": [32, 32], "realisations": R, "t_end": 10.0,
                  "launch": {"threads": thr, "ctas_per_sm": cps}}, res["batched"][1] * 1e3,
                 {"plain": {"value": res["plain"][0], "seconds": res["plain"][1]},
                  "wide": {"value": res["wide"][0], "seconds": res["wide"][1]},
                  "batched_over_plain": res["batched"][0] / res["plain"][0],
                  "wide_over_plain": res["wide"][0] / res["plain"][0],
                  "same_stats": "bit-identical final states (plain vs batched)" if same else "MISMATCH",
                  "bit_identical": same})


def ensemble(args, rank, world):
    """4096 random heterogeneous instances (side 16..128, 4..12 species, 8..32
    reactions), t = 5, in one persistent kernel (launch shape from the autotuner),
    against the reference's structure -- one solver per instance, a wait after every
    launch -- timed on a sample of the instances and compared per cell-step.  A plain
    instance runs the same random streams as in the batch, so its final state must be
    bit-identical to the batched one (checked for every sampled instance).  The
    persistent kernel is warmed up on a 64-instance ensemble, then the whole ensemble
    runs once, timed (one launch of 20 s: launch overheads do not show)."""
    import torch
    from .ensemble import Ensemble, autotune, random_ensemble
    from .solver import Solver
    n = int(getattr(args, "instances", 4096))
    n = max(1, n)
    specs = random_ensemble(n, seed=2024, max_time=5.0)
    (thr, cps), tune = autotune(specs)
    warm = Ensemble(specs[:64])
    warm.configure(thr, cps)
    ws = warm.alloc_state()
    for _ in range(max(1, int(getattr(args, "warmup", 3)))):
        warm.init_poisson(ws)
        warm.run(ws)
    torch.cuda.synchronize()
    del warm, ws
    ens = Ensemble(specs)
    ens.configure(thr, cps)
    state = ens.alloc_state()
    ens.init_poisson(state)
    a, b = _events()
    a.record()
    ens.run(state)                    # graph capture (no work) + one replay
    b.record()
    torch.cuda.synchronize()
    t = a.elapsed_time(b) / 1e3
    status, steps, _ = ens.results()
    cs = ens.cell_steps(steps)
    batched = cs / t
    # plain: the reference's structure on a sample of the instances
    k = int(getattr(args, "plain_sample", 24))
    pick = np.random.default_rng(1).choice(n, size=min(k, n), replace=False)
    pcs, pt, same = 0, 0.0, True
    for i in pick:
        sp = specs[int(i)]
        with Solver(sp.model, realisations=1, seed=sp.seed, sync_each_launch=True) as s:
            s.init_poisson(sp.lam)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            _, _, nsteps = s.solve(count_only=True)
            torch.cuda.synchronize()
            pt += time.perf_counter() - t0
            pcs += sp.model.area * nsteps
            fin = s.get_state()[0]
        same = same and nsteps == int(steps[int(i)]) and \
            np.array_equal(fin, ens.instance_state(state, int(i)).cpu().numpy())
    plain = pcs / pt
    return _base(args, world, batched, "cell-steps/s", "ensemble_4096_random_instances_t5",
                 {"instances": n, "launch": {"threads": thr, "ctas_per_sm": cps}, "autotune_ms": tune.get("ms")},
                 t * 1e3,
                 {"plain": {"value": plain, "sample_instances": len(pick), "seconds": pt},
                  "batched_over_plain": batched / plain, "instances_with_status": int((status != 0).sum()),
                  "same_stats": ("bit-identical final states on the sampled instances" if same else "MISMATCH"),
                  "bit_identical": bool(same), "cell_steps": cs,
                  # the graph holds two memset nodes and one k_ensemble launch
                  "gpu_launches": 1})


def lotka_volterra(args, rank, world):
    """Inhomogeneous drift-diffusion SSA, 512 x 512, Lotka-Volterra, lognormal D,
    sinusoidal drift, 256 realisations; timed over t in [0, t_sample]."""
    import torch
    from .model import lotka_volterra_model
    from .solver import Solver
    t_sample = float(getattr(args, "t_sample", 0.5))
    m = lotka_volterra_model(width=512, max_time=t_sample)
    R = 256
    with Solver(m, realisations=R, seed=1234) as s:
        s.init_poisson([50.0, 50.0])
        torch.cuda.synchronize()
        a, b = _events()
        a.record()
        _, _, steps = s.solve(count_only=True)
        b.record()
        torch.cuda.synchronize()
        t = a.elapsed_time(b) / 1e3
        st = s.status()
    cs = m.area * R * steps
    return _base(args, world, cs / t, "cell-steps/s", "lotka_volterra_512x512_256real",
                 {"grid": [512, 512], "realisations": R, "t_sample": t_sample, "steps": steps},
                 t / max(steps, 1) * 1e3, {"status_nonzero": int((st != 0).sum())})


def particles(args, rank, world):
    """2^22 particles on 1024 x 1024 cells: Brownian step (D = 0.5, drift (0.1, 0)),
    radix-sort binning + exclusive scan, in-cell A+B->0 (p = 0.05); K steps timed."""
    import torch
    from .individual import Particles, uniform_particles
    n, G = 1 << 22, 1024
    x, y, sp = uniform_particles(n, G, seed=1234)
    p = Particles(n, G, D=0.5, vx=0.1, vy=0.0, dt=1.0, p_react=0.05, seed=1234)
    p.set(x, y, sp, step=0)
    p.step(args.warmup)
    torch.cuda.synchronize()
    a, b = _events()
    x0, _, _ = p.get()
    n0 = len(x0)
    a.record()
    p.step(args.steps)
    b.record()
    torch.cuda.synchronize()
    t = a.elapsed_time(b) / 1e3
    x1, _, _ = p.get()
    ps = (n0 + len(x1)) / 2 * args.steps
    # kernels per step for the 20-bit cell keys: move, two 10-bit onesweep passes (the
    # last counts the cells), react + compact
    launches = 4 * args.steps
    # Roofline of the whole step (the kernels run inside one library call): the bytes
    # that must move at least once per particle -- move 24 (read x, y; write x, y, key,
    # index), two sort passes 2 x 16 (the cell counts come with the last), react +
    # compact 4 index + 1 species + 8 position read, 9 written -- plus 12 B per cell
    # (count written and read, start written)
    alg = 78.0 * ps / args.steps + 12.0 * G * G
    ach = alg / (t / args.steps) / 1e9
    peak, peak_kind = _peaks()
    extra = {"particles_left": len(x1), "dtype": "f32+u32", "gpu_launches": launches,
             "roofline": {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                          "peak_kind": peak_kind, "traffic": None, "scope": "whole step",
                          "algorithmic_bytes_per_step": alg}}
    return _base(args, world, ps / t, "particle-steps/s", "particles_2^22_1024x1024",
                 {"particles": n, "grid": [G, G], "steps_timed": args.steps}, t / args.steps * 1e3, extra)


def population(args, rank, world):
    """Individual bookkeeping (maintainPopulation): 1024 x 1024 cells holding Poisson(4)
    individuals (about 4.2e6) sorted by cell, a free-id pool of 2^21; every step each
    cell's target count moves by -1, 0 or +1.  Timed: one gpgmp_population_maintain
    call per step on resident buffers (the list alternates between two buffer sets).

    Roofline: the bytes the operation must move at least once -- read keys and ids,
    write the new keys and ids (16 B per individual), read start, count and goal and
    write the new start (16 B per cell), read and write the pool (8 B per entry)."""
    import ctypes as C
    import os
    import sys
    import torch
    from .individual import _call, _ptr, _stream
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from bench import load_peaks
    G, mean, npool0 = 1024, 4.0, 1 << 21
    ncells = G * G
    rng = np.random.default_rng(1234)
    counts = rng.poisson(mean, ncells).astype(np.uint32)
    n = int(counts.sum())
    keys = np.repeat(np.arange(ncells, dtype=np.uint32), counts)
    perm = rng.permutation(n + npool0).astype(np.uint32)
    start = np.concatenate([[0], np.cumsum(counts)[:-1]]).astype(np.uint32)
    dev = torch.device("cuda", torch.cuda.current_device())
    cap = n + npool0
    tot = lambda a: torch.from_numpy(a.view(np.int32)).to(dev)
    bufs = []
    for _ in range(2):
        bufs.append({"keys": torch.empty(cap, dtype=torch.int32, device=dev),
                     "ids": torch.empty(cap, dtype=torch.int32, device=dev),
                     "pool": torch.empty(cap, dtype=torch.int32, device=dev),
                     "start": torch.empty(ncells, dtype=torch.int32, device=dev)})
    bufs[0]["keys"][:n] = tot(keys)
    bufs[0]["ids"][:n] = tot(perm[:n].copy())
    bufs[0]["pool"][:npool0] = tot(perm[n:].copy())
    bufs[0]["start"][:] = tot(start)
    count = tot(counts)
    nsteps = args.warmup + args.steps
    goals = []
    g = counts.astype(np.int64)
    for _ in range(nsteps):
        g = np.maximum(g + rng.integers(-1, 2, ncells), 0)
        goals.append(tot(g.astype(np.int32)))
    sb = C.c_size_t(0)
    _call("gpgmp_population_scratch_bytes", cap, ncells, C.byref(sb))
    scratch = torch.empty(sb.value, dtype=torch.uint8, device=dev)
    state = {"n": n, "npool": npool0, "count": count}
    na, npo = C.c_int64(0), C.c_int64(0)
    moved = []

    def step(k):
        src, dst = bufs[k % 2], bufs[(k + 1) % 2]
        _call("gpgmp_population_maintain", _ptr(src["keys"]), _ptr(src["ids"]), state["n"], _ptr(src["start"]),
              _ptr(state["count"]), _ptr(goals[k]), ncells, _ptr(src["pool"]), state["npool"], 1234, k,
              _ptr(dst["keys"]), _ptr(dst["ids"]), cap, _ptr(dst["pool"]), cap, _ptr(dst["start"]),
              C.byref(na), C.byref(npo), _ptr(scratch), scratch.numel(), _stream())
        moved.append(16 * (state["n"] + na.value) // 2 + 16 * ncells + 8 * (state["npool"] + npo.value) // 2)
        state["n"], state["npool"], state["count"] = na.value, npo.value, goals[k]

    for k in range(args.warmup):
        step(k)
    torch.cuda.synchronize()
    moved.clear()
    n_before = state["n"]
    a, b = _events()
    a.record()
    for k in range(args.warmup, nsteps):
        step(k)
    b.record()
    torch.cuda.synchronize()
    t = a.elapsed_time(b) / 1e3
    # the last list must hold exactly the last goal, still sorted by cell
    last = bufs[nsteps % 2]
    kk = last["keys"][:state["n"]].cpu().numpy().view(np.uint32)
    ok = bool(np.all(np.diff(kk.astype(np.int64)) >= 0) and
              np.array_equal(np.bincount(kk, minlength=ncells), goals[-1].cpu().numpy()))
    inds = (n_before + state["n"]) / 2 * args.steps
    launches_per_call = 2     # k_pop_plan, k_pop_move
    alg = sum(moved) / args.steps
    peak, peak_kind = load_peaks()
    ach = alg / (t / args.steps) / 1e9
    return _base(args, world, inds / t, "individuals/s", "population_1024x1024_poisson4_pool2^21",
                 {"grid": [G, G], "individuals": n, "pool": npool0, "goal_change": "U{-1,0,1} per cell per step",
                  "l2": "inputs larger than L2 (about 70 MB read + 70 MB written per step, ping-pong buffers)"},
                 t / args.steps * 1e3,
                 {"dtype": "u32", "invariants_ok": ok, "gpu_launches": launches_per_call * args.steps,
                  "roofline": {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                               "peak_kind": peak_kind, "traffic": None,
                               "algorithmic_bytes_per_step": alg}})


def individuals(args, rank, world):
    """Individual species in the drift-diffusion solver: 256 x 256 cells, 4 individuals
    per cell (262,144, the reference's c_maxNumIndividuals), each with its own
    diffusivity (0.3..0.7) and drift (-0.2..0.2); one step = one x and one y sweep of
    every individual (one kernel moves it and folds its cell's count and fields in,
    a second writes the counts to the state and takes the time step, which is read
    back; the list is sorted only when read).  Unit: individual-sweeps/s.

    Roofline: per individual and sweep the bytes that must move at least once -- read
    key, id and four properties, write the key (28 B) -- plus 24 B per cell (count and
    four fields written and read, the state written)."""
    import torch
    from . import _lib
    from .model import DiffusionModel
    from .solver import Solver
    W = 256
    m = DiffusionModel(width=W, height=W, physical_length=float(W), solver=_lib.STOCHASTIC_INHOMOGENEOUS)
    m.add_species("A", 0.0, individual=True)
    m.drift_method = _lib.DRIFT_HOMOGENEOUS
    m.drift_params = [0.5, 0.5, 0.0, 0.0] + [0.0] * 4
    m.individual_capacity = 1 << 19
    st = np.full((1, 1, W, W), 4, np.int32)
    n = int(st.sum())
    rng = np.random.default_rng(1234)
    props = np.stack([rng.uniform(0.3, 0.7, n), rng.uniform(0.3, 0.7, n), rng.uniform(-0.2, 0.2, n),
                      rng.uniform(-0.2, 0.2, n)]).astype(np.float32)
    with Solver(m, realisations=1, seed=1234) as s:
        s.set_state(st)
        s.set_individual_properties(0, props)
        seed = 1
        t = 0.0

        def one_step(seed, t):
            dx, dy = s.timesteps()
            t = t + float(max(dx[0], dy[0]))
            return s.diffuse(0, t, seed), t

        for _ in range(args.warmup):
            seed, t = one_step(seed, t)
        torch.cuda.synchronize()
        a, b = _events()
        a.record()
        for _ in range(args.steps):
            seed, t = one_step(seed, t)
        b.record()
        torch.cuda.synchronize()
        tsec = a.elapsed_time(b) / 1e3
        n_end = s.individual_count(0)
    sweeps = 2 * args.steps
    value = n * sweeps / tsec
    alg = 28 * n + 24 * W * W                           # per sweep
    ach = alg / (tsec / sweeps) / 1e9
    peak, peak_kind = _peaks()
    return _base(args, world, value, "individual-sweeps/s", "individuals_256x256_262144",
                 {"grid": [W, W], "individuals": n, "steps_timed": args.steps, "sweeps_per_step": 2},
                 tsec / args.steps * 1e3,
                 {"dtype": "u32+f32", "individuals_left": n_end,
                  # per sweep: the fused move, the counts with the time step
                  "gpu_launches": 2 * sweeps,
                  "roofline": {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                               "peak_kind": peak_kind, "traffic": None, "algorithmic_bytes_per_sweep": alg}})


def _peaks():
    import os
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from bench import load_peaks
    return load_peaks()


def _profile_figures(name):
    """`key: value` lines at the top of a profile summary (measured DRAM traffic per
    launch, from its ncu capture)."""
    import os
    path = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "profiles", name)
    out = {}
    if os.path.exists(path):
        for ln in open(path):
            k, sep, v = ln.partition(":")
            if sep and k.endswith("_bytes_per_launch"):
                try:
                    out[k.strip()] = float(v)
                except ValueError:
                    pass
    return out


def scan_sort(args, rank, world):
    """The individual-particle primitives on their own, through the C ABI: exclusive
    scan of 2^27 uint32 values (512 MB in, 512 MB out: larger than L2, so no flush is
    needed between calls) and stable sorts of 2^24 (key, value) pairs with 20-bit keys
    (two 10-bit passes) and 32-bit keys (four 8-bit passes).  Unit of the line's value:
    scanned values/s; the sorts are reported beside it in keys/s.

    Roofline (scan): 8 B per value (read, write); (sort) 16 B per key and pass (read
    key and value, write key and value).  Library comparators, timed the same way on
    the same inputs: torch.cumsum (int32) beside the scan, torch.sort(stable=True)
    (int32 keys with int64 indices) beside each sort."""
    import torch
    from . import individual as ind
    dev = "cuda"
    gen = torch.Generator(device=dev)
    gen.manual_seed(1234)
    n = 1 << 27
    x = torch.randint(0, 16, (n,), dtype=torch.int32, device=dev, generator=gen)
    out = torch.empty_like(x)
    scr = ind.scan_scratch(n)

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        a, b = _events()
        a.record()
        for _ in range(args.steps):
            fn()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / 1e3 / args.steps

    t_scan = timed(lambda: ind._call("gpgmp_exclusive_scan_u32", ind._ptr(x), ind._ptr(out), n, ind._ptr(scr),
                                     scr.numel(), ind._stream()))
    # library comparator: torch.cumsum on the same int32 values (inclusive, int32 out)
    lib_out = torch.empty_like(x)
    t_cumsum = timed(lambda: torch.cumsum(x, 0, dtype=torch.int32, out=lib_out))
    del lib_out
    peak, peak_kind = _peaks()
    figs = _profile_figures("scan_sort_2p27_2p24.md")
    ns = 1 << 24
    sorts = {}
    for bits, passes in ((20, 2), (32, 4)):
        k = torch.randint(0, 1 << bits, (ns,), dtype=torch.int64, device=dev, generator=gen).to(torch.int32)
        v = torch.arange(ns, dtype=torch.int32, device=dev)
        ko, vo = torch.empty_like(k), torch.empty_like(v)
        sscr = ind.sort_scratch(ns, bits)
        t = timed(lambda: ind._call("gpgmp_sort_pairs_u32", ind._ptr(k), ind._ptr(v), ind._ptr(ko), ind._ptr(vo), ns,
                                    bits, ind._ptr(sscr), sscr.numel(), ind._stream()))
        ach = 16.0 * passes * ns / t / 1e9
        # library comparator on the same keys: torch.sort(stable=True) (int32 keys, int64
        # indices as the values: 12 B per key moved each pass instead of 8)
        t_lib = timed(lambda: torch.sort(k, stable=True))
        # the library's digit width: 10 bits where that saves a pass, else 8
        digit = 10 if 16 < bits <= 30 and (bits + 9) // 10 < (bits + 7) // 8 else 8
        pass_traffic = figs.get(f"sort{digit}_pass_traffic_bytes_per_launch")
        sorts[f"keys_{bits}bit"] = {"pairs": ns, "passes": passes, "ms_per_sort": t * 1e3, "keys_per_s": ns / t,
                                    "roofline": {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s",
                                                 "frac": ach / peak, "peak_kind": peak_kind,
                                                 "traffic_per_pass": pass_traffic,
                                                 "algorithmic_bytes_per_pass": 16 * ns},
                                    "torch_sort_stable_ms": t_lib * 1e3}
        del k, v, ko, vo, sscr
    ach = 8.0 * n / t_scan / 1e9
    return _base(args, world, n / t_scan, "values/s", "scan_2^27_u32_sort_2^24_pairs",
                 {"scan_values": n, "sort_pairs": ns, "l2": "inputs larger than L2 (scan)"}, t_scan * 1e3,
                 {"dtype": "u32", "sorts": sorts, "torch_cumsum_int32_ms": t_cumsum * 1e3,
                  # per timed scan: one scan kernel; per sort: histogram + one kernel per pass
                  "gpu_launches": args.steps * (1 + (1 + 2) + (1 + 4)),
                  "roofline": {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                               "peak_kind": peak_kind, "traffic": figs.get("scan_traffic_bytes_per_launch"),
                               "algorithmic_bytes_per_scan": 8 * n}})


def run(args, rank, world):
    table = {"ssa_plain": ssa_plain, "lotka_volterra": lotka_volterra, "particles": particles,
             "ensemble": ensemble, "population": population, "individuals": individuals, "scan_sort": scan_sort}
    if args.workload not in table:
        raise SystemExit(f"unknown workload {args.workload}; one of gray_scott, {', '.join(table)}")
    return table[args.workload](args, rank, world)
