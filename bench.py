"""Benchmark of the B200 GPGMP hot path.

Default workload (one JSON line): deterministic Gray-Scott reaction-diffusion,
256 x 256 periodic lattice, FP32, F=0.04, k=0.06, Du=0.16, Dv=0.08, dt=1, 10,000
explicit steps (synthetic seeded initial state).  A bench step is one full
10,000-step forward solve; value = cell-steps/s with the state resident in HBM;
e2e = the same through the C ABI call with host buffers (copies inside the timed
region); adjoint_forward_ratio = time of the gradient (adjoint with checkpointing,
recomputation included) over the time of one forward solve.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload gray_scott|ssa_plain|lotka_volterra|ensemble|particles|population|individuals|scan_sort]

Multi-GPU: every rank runs its own replica (the path does not shard: replicas
only); value = total cell-steps of all ranks / max over ranks of the time.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "cell-steps/s per B200, batched vs plain at same stats; adjoint/forward time ratio"


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """SM clock and clock-event (throttle) reasons of this process's GPU, read through
    NVML every 10 ms from a thread while the timed region runs (read-only queries; the
    GPU is found by its PCI bus id, so a remapped CUDA_VISIBLE_DEVICES still names the
    right board).  Falls back to nvidia-smi at 200 ms where NVML is unavailable."""

    # NVML clock-event reason bits (nvml.h: nvmlClocksEventReason*)
    REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
               ("sw_power_cap", 0x4))

    def __init__(self, index: int = 0, period: float = 0.01):
        self.index = index
        self.period = period
        self.samples = []          # (sm_mhz, max_mhz, reason bits)
        self.proc = None
        self.lines = []
        self._stop = threading.Event()
        self._nvml = None

    def _handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        pr = torch.cuda.get_device_properties(torch.cuda.current_device())
        bus = "%08X:%02X:%02X.0" % (pr.pci_domain_id, pr.pci_bus_id, pr.pci_device_id)
        return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)

    def _poll(self, nv, h):
        mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        get_reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            nv.nvmlDeviceGetCurrentClocksThrottleReasons
        while True:
            try:
                self.samples.append((float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)), float(mx),
                                     int(get_reasons(h))))
            except Exception:
                pass
            if self._stop.wait(self.period):
                break

    def __enter__(self):
        try:
            nv, h = self._handle()
            self._nvml = nv
            self.t = threading.Thread(target=self._poll, args=(nv, h), daemon=True)
            self.t.start()
            t0 = time.perf_counter()
            while not self.samples and time.perf_counter() - t0 < 1.0:   # first sample before the work
                time.sleep(0.001)
            return self
        except Exception:
            self._nvml = None
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self._nvml is not None:
            self._stop.set()
            self.t.join(timeout=5)
            try:
                self._nvml.nvmlShutdown()
            except Exception:
                pass
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        mhz, mx, reasons = [], None, set()
        for sm, m, bits in self.samples:
            mhz.append(sm)
            mx = m
            for nm, bit in self.REASONS:
                if bits & bit:
                    reasons.add(nm)
        names = [nm for nm, _ in self.REASONS]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                mhz.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(mhz)) if mhz else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(mhz), "source": "nvml" if self.samples else "nvidia-smi"}


def dist_setup(args):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl != "reference":
        torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        backend = "nccl" if args.impl != "reference" else "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x: float, world: int) -> float:
    """The largest x over the ranks (the job's time is its slowest rank's)."""
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(units_per_rank: float, seconds: float, world: int) -> float:
    """Whole-job throughput of independent replicas: every rank's units over the
    slowest rank's time."""
    return units_per_rank * world / max_over_ranks(seconds, world)


def flush_l2(buf):
    buf.add_(1)


# ---------------------------------------------------------------------------
# Gray-Scott (deterministic reaction-diffusion + adjoint)
# ---------------------------------------------------------------------------

def bench_gray_scott(args, rank, world):
    import torch
    from inchman_b200 import gray_scott as gs
    cfg = gs.GrayScottConfig()
    n, steps = cfg.n, cfg.steps
    cell_steps = n * n * steps
    u0h, v0h = cfg.initial_state(np.float32)
    dev = torch.device("cuda")
    u0 = torch.tensor(u0h, device=dev)
    v0 = torch.tensor(v0h, device=dev)
    p = cfg.params()
    kernel = forward_kernel(n)    # what the automatic choice (variant 0) runs here
    l2 = torch.zeros(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MB > 126 MB L2
    stream = torch.cuda.current_stream()
    for _ in range(args.warmup):
        gs.forward(u0, v0, p)
    torch.cuda.synchronize()
    # ---- device-resident forward: K solves, each timed with events, L2 flushed between
    times = []
    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        barrier(world)
        torch.cuda.synchronize()
        for _ in range(args.steps):
            flush_l2(l2)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            gs.forward(u0, v0, p)
            b.record(stream)
            times.append((a, b))
        torch.cuda.synchronize()
        barrier(world)
    per = [a.elapsed_time(b) / 1e3 for a, b in times]
    t_total = max_over_ranks(sum(per), world)
    value = cell_steps * args.steps * world / t_total      # replica_value with the reduced time
    t_launch = sum(per) / len(per)
    # ---- batched: the nine solves of the central finite-difference check (base and
    # +-h in F, k, Du, Dv), one 16-CTA cluster each in one launch, against the same
    # nine solved one after another
    h = 1e-3
    members = [[cfg.F, cfg.k, cfg.Du, cfg.Dv, 0.0, 0.0]]
    for q in range(4):
        for sgn in (1.0, -1.0):
            m_ = list(members[0])
            m_[q] += sgn * h
            members.append(m_)
    B = len(members)
    U0 = u0.unsqueeze(0).repeat(B, 1, 1).contiguous()
    V0 = v0.unsqueeze(0).repeat(B, 1, 1).contiguous()
    gs.forward_batch(U0, V0, p, member_params=members)
    torch.cuda.synchronize()
    flush_l2(l2)
    ba, bb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ba.record(stream)
    gs.forward_batch(U0, V0, p, member_params=members)
    bb.record(stream)
    torch.cuda.synchronize()
    t_batch = ba.elapsed_time(bb) / 1e3
    singles = [gs.GrayScottConfig(F=m_[0], k=m_[1], Du=m_[2], Dv=m_[3]).params() for m_ in members]
    flush_l2(l2)
    sa, sb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    sa.record(stream)
    for ps in singles:
        gs.forward(u0, v0, ps)
    sb.record(stream)
    torch.cuda.synchronize()
    t_plain9 = sa.elapsed_time(sb) / 1e3
    batched = {"members": B, "what": "central FD check: base and +-1e-3 in F, k, Du, Dv",
               "lattices_at_once": gs.batch_capacity(n),
               "value": B * cell_steps / t_batch, "unit": "cell-steps/s", "seconds": t_batch,
               "plain_seconds": t_plain9, "batched_over_plain": t_plain9 / t_batch}
    # ---- end to end through the C ABI with pinned host buffers
    pu = torch.from_numpy(u0h).pin_memory()
    pv = torch.from_numpy(v0h).pin_memory()
    ou = torch.empty_like(pu).pin_memory()
    ov = torch.empty_like(pv).pin_memory()
    nu, nv, nou, nov = pu.numpy(), pv.numpy(), ou.numpy(), ov.numpy()
    import ctypes as C
    fh = gs._fn("gpgmp_gs_forward_host")
    for _ in range(max(1, args.warmup)):
        fh(C.byref(p), nu.ctypes.data_as(C.c_void_p), nv.ctypes.data_as(C.c_void_p), nou.ctypes.data_as(C.c_void_p),
           nov.ctypes.data_as(C.c_void_p))
    torch.cuda.synchronize()
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        rc = fh(C.byref(p), nu.ctypes.data_as(C.c_void_p), nv.ctypes.data_as(C.c_void_p),
                nou.ctypes.data_as(C.c_void_p), nov.ctypes.data_as(C.c_void_p))
        if rc != 0:
            raise RuntimeError("gpgmp_gs_forward_host failed")
    t_e2e = max_over_ranks(time.perf_counter() - t0, world)
    e2e = cell_steps * args.steps * world / t_e2e
    # ---- adjoint / forward ratio (gradient of the snapshot loss)
    ckb, _ = gs.buffer_sizes(p, 4)
    ck = torch.empty(ckb // 4, dtype=torch.float32, device=dev)
    ut, vt = gs.forward(u0, v0, gs.GrayScottConfig(F=0.042).params())
    GS = gs.GrayScott()
    th = torch.tensor(cfg.theta(), dtype=torch.float64, device=dev, requires_grad=True)

    def grad_once():
        u, v = GS.apply(u0, v0, th, steps, cfg.dt, 0)        # automatic interval: 100 steps
        loss = ((u - ut) ** 2 + (v - vt) ** 2).sum()
        loss.backward()
        return loss

    for _ in range(2):
        grad_once()
    torch.cuda.synchronize()
    ga, gb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    nrep = max(1, min(args.steps, 5))
    ga.record(stream)
    for _ in range(nrep):
        grad_once()
    gb.record(stream)
    torch.cuda.synchronize()
    t_grad = ga.elapsed_time(gb) / 1e3 / nrep
    # forward + backward over forward-only time
    ratio = t_grad / t_launch
    # the same ratio in float64, the precision whose gradient meets 1e-4 against
    # finite differences and equals the oracle's float64 CPU adjoint
    u064, v064 = u0.double(), v0.double()
    ut64, vt64 = ut.double(), vt.double()

    def grad64_once():
        u, v = GS.apply(u064, v064, th, steps, cfg.dt, 0)    # automatic interval: 25 steps
        loss = ((u - ut64) ** 2 + (v - vt64) ** 2).sum()
        loss.backward()
        return loss

    gs.forward(u064, v064, p)
    grad64_once()
    torch.cuda.synchronize()
    fa, fb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    nrep64 = max(1, min(args.steps, 3))
    fa.record(stream)
    for _ in range(nrep64):
        gs.forward(u064, v064, p)
    fb.record(stream)
    torch.cuda.synchronize()
    t_fwd64 = fa.elapsed_time(fb) / 1e3 / nrep64
    fa.record(stream)
    for _ in range(nrep64):
        grad64_once()
    fb.record(stream)
    torch.cuda.synchronize()
    t_grad64 = fa.elapsed_time(fb) / 1e3 / nrep64
    peak, peak_kind = load_peaks()
    alg_bytes = 16.0 * cell_steps
    achieved = alg_bytes / t_launch / 1e9
    traffic = None
    prof = os.path.join(ROOT, "profiles", "gray_scott_forward_256x256.md")
    if os.path.exists(prof):
        for ln in open(prof):
            if ln.startswith("traffic_bytes_per_launch:"):
                traffic = float(ln.split(":")[1])
    clocks = clk.summary()
    line = {
        "metric": METRIC, "value": value, "unit": "cell-steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_total / args.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
        "config": {"workload": "gray_scott_256x256_periodic_fp32_10000_steps", "lattice": [n, n],
                   "explicit_steps_per_bench_step": steps, "cell_steps_per_bench_step": cell_steps,
                   "F": cfg.F, "k": cfg.k, "Du": cfg.Du, "Dv": cfg.Dv, "dt": cfg.dt,
                   "l2": "flushed between timed iterations (256 MB write)",
                   "parallelism": f"replicas x{world}"},
        "adjoint_forward_ratio": ratio,
        "adjoint_forward_ratio_f64": t_grad64 / t_fwd64,
        "gradient_ms": t_grad * 1e3,
        "gradient_ms_f64": t_grad64 * 1e3, "forward_ms_f64": t_fwd64 * 1e3,
        "checkpoint_every": {"f32": 100, "f64": 25},
        "batched_fd_solves": batched,
        "e2e": {"value": e2e, "unit": "cell-steps/s", "h2d_bytes_per_step": 2 * n * n * 4,
                "d2h_bytes_per_step": 2 * n * n * 4},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "peak_source": peak_kind,
                     "note": kernel_note(kernel),
                     "sm_bound": sm_bound(t_launch, steps, n, clocks.get("sm_mhz"), kernel)},
        "kernel": kernel,
        "gpu_launches": args.steps,   # one forward-kernel launch per timed solve
        "clocks": clocks,
    }
    if rank == 0 and world == 1:
        line["cpu_baseline"] = cpu_baseline_gray_scott(cfg)
        if not getattr(args, "headline_only", False):
            paths = path_blocks(args)
            line["paths"] = paths
            line["batched_over_plain"] = {"c4_ensemble_4096": paths["c4_ensemble_4096"]["batched_over_plain"],
                                          "c1_ssa_plain_32x32": paths["c1_ssa_plain_32x32"]["batched_over_plain"],
                                          "same_stats": "bit-identical final states, plain vs batched"}
    return line


def forward_kernel(n):
    """The float32 forward kernel that the automatic choice runs for an n x n lattice
    on this GPU: its variant, 16-CTA clusters, SMs and rows computed per step (band
    plus ghost rows for the multi-cluster kernel)."""
    from inchman_b200 import gray_scott as gs
    v = gs.auto_variant(n)
    if v in gs.MULTI_CLUSTER:
        c, g = gs.MULTI_CLUSTER[v]
        return {"variant": v, "name": f"k_gs_forward_mc<{n},{c},{g},{(n // c + 2 * g) // 16}>", "clusters": c,
                "ghost_rows": g, "sms": 16 * c, "rows_per_step": n + 2 * g * c}
    if v > 10:
        return {"variant": v, "name": f"k_gs_forward_rr<{n},{v - 10}>", "clusters": 1, "ghost_rows": 0, "sms": 16,
                "rows_per_step": n}
    return {"variant": v, "name": "shared-memory column walk", "clusters": 1, "ghost_rows": 0, "sms": 16,
            "rows_per_step": n}


def kernel_note(kernel):
    c, g = kernel["clusters"], kernel["ghost_rows"]
    if c > 1:
        return (f"16 B/cell-step algorithmic; the lattice stays in the registers of {c} 16-CTA clusters "
                f"({16 * c} of 148 SMs; each cluster its band plus {g} ghost rows per side, swapped through "
                f"global memory every {g} steps), so DRAM traffic is the initial read, the final write and "
                f"the ghost-row swaps")
    return ("16 B/cell-step algorithmic; the lattice stays in the registers of one 16-CTA cluster "
            "(16 of 148 SMs), so DRAM traffic is the initial read and final write only")


def sm_bound(t_solve, steps, n, clock_mhz, kernel, ops_per_cell=18):
    """The compute bound of the forward solve on the SMs it occupies: 18 FP32 lane
    operations per cell-step (an FMA counts once), 128 FP32 lanes per SM at the median
    SM clock sampled during the timed solves, over the lattice's n x n cells
    (`frac`) and over the rows the kernel actually computes, ghost rows included
    (`frac_with_ghost_rows`)."""
    clk = float(clock_mhz or 1965.0) * 1e6
    sms = kernel["sms"]
    bound = n * n * ops_per_cell / (sms * 128 * clk)
    bound_all = kernel["rows_per_step"] * n * ops_per_cell / (sms * 128 * clk)
    per = t_solve / steps
    return {"sms_used": sms, "fp32_ops_per_cell_step": ops_per_cell, "sm_clock_hz": clk,
            "bound_us_per_step": bound * 1e6, "achieved_us_per_step": per * 1e6, "frac": bound / per,
            "rows_computed_per_step": kernel["rows_per_step"], "frac_with_ghost_rows": bound_all / per}


def path_blocks(args):
    """The other hot-path workloads, each measured once in the default line (a bounded
    form of bench.py --workload <name>): C1 plain vs batched SSA, C3 drift-diffusion
    SSA (t in [0, 0.5]), C4 batched ensemble vs plain, C5 particle binning, and the
    scan / sort primitives."""
    from types import SimpleNamespace
    from inchman_b200 import workloads
    ns = SimpleNamespace(steps=max(3, min(args.steps, 20)), warmup=max(3, args.warmup), instances=4096,
                         plain_sample=24, t_sample=0.5, workload="")
    drop = {"metric", "n_gpus", "steps", "warmup", "higher_is_better", "scaling", "vs_baseline", "data"}
    out = {}
    for key, fn in (("c1_ssa_plain_32x32", workloads.ssa_plain), ("c3_drift_diffusion_512x512", workloads.lotka_volterra),
                    ("c4_ensemble_4096", workloads.ensemble), ("c5_particles_2p22", workloads.particles),
                    ("scan_sort", workloads.scan_sort)):
        t0 = time.perf_counter()
        d = fn(ns, 0, 1)
        out[key] = {k: v for k, v in d.items() if k not in drop}
        out[key]["wall_s"] = time.perf_counter() - t0
    return out


def cpu_baseline_particles(steps=3):
    """The oracle's replay of the particle step (OpenMP C) on the host cores: a bounded
    sample of three steps of the same 2^22 seeded particles as the GPU workload."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    from inchman_b200.individual import uniform_particles
    G = 1024
    x, y, sp = uniform_particles(1 << 22, G, seed=1234)
    n = len(x)
    t0 = time.perf_counter()
    m = oracle.orc().orc_particles_run(n, oracle.ptr(x), oracle.ptr(y), oracle.ptr(sp), G, 0.5, 0.1, 0.0, 1.0, 0.05,
                                       1234, 0, steps)
    dt = time.perf_counter() - t0
    return {"value": (n + m) / 2 * steps / dt, "unit": "particle-steps/s", "cores": os.cpu_count(), "kind": "port",
            "sample": f"{steps} steps of the same {n} particles (oracle, OpenMP)"}


def _gs_cpu_sample(explicit_steps: int, reps: int, warm: int = 1):
    """Runs in a child process that imports only numpy and the oracle (no torch, no CUDA
    context, one OpenMP runtime): times `reps` forward solves of `explicit_steps` steps
    of the Gray-Scott lattice with the oracle's float32 port (vectorised C, OpenMP over
    rows) after `warm` untimed ones; prints one JSON line."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    from inchman_b200.gray_scott import GrayScottConfig
    cfg = GrayScottConfig()
    u0, v0 = cfg.initial_state(np.float32)
    L = oracle.orc()

    def one():
        u, v = u0.copy(), v0.copy()
        L.orc_gs_forward_f32(cfg.n, explicit_steps, cfg.F, cfg.k, cfg.Du, cfg.Dv, cfg.vx, cfg.vy, cfg.dt,
                             oracle.ptr(u), oracle.ptr(v))

    for _ in range(warm):
        one()
    times = []
    for _ in range(reps):
        t0 = time.perf_counter()
        one()
        times.append(time.perf_counter() - t0)
    print(json.dumps({"times": times, "threads": os.environ.get("OMP_NUM_THREADS") or os.cpu_count()}), flush=True)


def gs_cpu_times(explicit_steps: int, reps: int, warm: int = 1):
    """Per-solve seconds of the CPU port, measured in a clean child process (the same
    measurement for the reported cpu_baseline and for the reference arm)."""
    env = dict(os.environ)
    env.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
    out = subprocess.run([sys.executable, os.path.abspath(__file__), "--gs-cpu-sample",
                          f"{explicit_steps},{reps},{warm}"], capture_output=True, text=True, env=env, check=True)
    d = json.loads(out.stdout.strip().splitlines()[-1])
    return d["times"], int(d["threads"])


# The CPU measures the whole 10,000-step solve, not a prefix of it: the port's speed
# changes along the trajectory (as v decays, many values become subnormal and the
# CPU's arithmetic on them is slow), so a shorter sample would not stand for the
# workload.  One solve takes about a second on a 16-core host.
CPU_SAMPLE_STEPS = 10_000


def cpu_baseline_gray_scott(cfg, reps=3):
    times, threads = gs_cpu_times(CPU_SAMPLE_STEPS, reps)
    t = sum(times)
    return {"value": cfg.n * cfg.n * CPU_SAMPLE_STEPS * reps / t, "unit": "cell-steps/s", "cores": threads,
            "kind": "port",
            "sample": f"{reps} full solves of the workload ({CPU_SAMPLE_STEPS} explicit steps of the 256x256 "
                      f"lattice) by the oracle's vectorised float32 port, bit-identical to the GPU kernel; "
                      f"OpenMP, {threads} threads, clean child process"}


def reference_gray_scott(args, rank, world):
    """The reference's CPU implementation of the path: the oracle's port of the explicit
    step (the reference's deterministic reaction kernel is code it generates per model,
    so the reference itself does not build for this network), all host threads; each
    bench step is one full solve of the workload (CPU_SAMPLE_STEPS explicit steps),
    timed in the same clean child process as the other arm's cpu_baseline."""
    from inchman_b200.gray_scott import GrayScottConfig
    cfg = GrayScottConfig()
    times, cores = gs_cpu_times(CPU_SAMPLE_STEPS, args.steps, warm=max(1, min(args.warmup, 2)))
    t = sum(times)
    v = cfg.n * cfg.n * CPU_SAMPLE_STEPS * args.steps / t
    return {"impl": "reference", "metric": METRIC, "value": v, "unit": "cell-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded)",
            "config": {"workload": "gray_scott_256x256_periodic_fp32_10000_steps",
                       "sample_explicit_steps_per_bench_step": CPU_SAMPLE_STEPS},
            "cpu_baseline": {"value": v, "unit": "cell-steps/s", "cores": cores, "kind": "port",
                             "sample": f"one full solve ({CPU_SAMPLE_STEPS} explicit steps of the 256x256 "
                                       f"lattice) per bench step"},
            "e2e": {"value": v, "unit": "cell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="gray_scott")
    ap.add_argument("--instances", type=int, default=4096, help="ensemble workload: number of instances")
    ap.add_argument("--plain-sample", type=int, default=24, help="ensemble workload: instances timed plain")
    ap.add_argument("--t-sample", type=float, default=0.5, help="lotka_volterra workload: simulated time")
    ap.add_argument("--headline-only", action="store_true",
                    help="default workload: only the Gray-Scott line, without the other paths' blocks")
    ap.add_argument("--gs-cpu-sample", default=None, help=argparse.SUPPRESS)
    args = ap.parse_args(argv)
    if args.gs_cpu_sample:
        k, reps, warm = (int(v) for v in args.gs_cpu_sample.split(","))
        _gs_cpu_sample(k, reps, warm)
        return 0
    args.warmup = max(args.warmup, 3) if args.impl != "reference" else args.warmup
    rank, world, local = dist_setup(args)
    if args.impl == "reference":
        if rank == 0:
            line = reference_gray_scott(args, rank, world)
            print(json.dumps(line), flush=True)
        return 0
    if args.workload == "gray_scott":
        line = bench_gray_scott(args, rank, world)
    else:
        from inchman_b200 import workloads
        line = workloads.run(args, rank, world)
        if args.workload == "particles" and rank == 0 and world == 1:
            line["cpu_baseline"] = cpu_baseline_particles()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
