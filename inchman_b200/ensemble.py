"""Batched ensembles of independent SSA + diffusion instances (one persistent
kernel, CUDA-graph replay), the random heterogeneous workload, and the
autotuner of the kernel's launch shape.

    ens = Ensemble.from_instances(instances)          # list of InstanceSpec
    state = ens.alloc_state(); ens.init_poisson(state)
    ens.run(state); status, steps = ens.results()
"""
from __future__ import annotations

import ctypes as C
import json
import os
import time
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from . import _lib
from .model import DiffusionModel

vp, i32, i64, f32, u32 = C.c_void_p, C.c_int32, C.c_int64, C.c_float, C.c_uint32
P = C.POINTER


class Instance(C.Structure):
    _fields_ = [("width", i32), ("num_species", i32), ("num_reactions", i32), ("species_offset", i32),
                ("reaction_offset", i32), ("boundary_mask", i32 * 4), ("physical_length", f32), ("p0", f32),
                ("max_time", f32), ("output_interval", f32), ("max_steps", i32), ("flags", i32),
                ("seed", u32), ("realisation", u32), ("max_snapshots", i32), ("reserved", i32),
                ("state_offset", i64), ("snapshot_offset", i64)]


_SIGS = {
    "gpgmp_ensemble_create": (C.c_int, [P(Instance), i32, P(f32), i64, P(f32), P(_lib.Reaction), i64, P(vp)]),
    "gpgmp_ensemble_destroy": (C.c_int, [vp]),
    "gpgmp_ensemble_configure": (C.c_int, [vp, i32, i32]),
    "gpgmp_ensemble_launch_shape": (C.c_int, [vp, P(i32), P(i32), P(i32)]),
    "gpgmp_ensemble_init_poisson": (C.c_int, [vp, vp, vp]),
    "gpgmp_ensemble_run": (C.c_int, [vp, vp, vp, vp]),
    "gpgmp_ensemble_results": (C.c_int, [vp, P(i32), P(i64), P(f32)]),
}
_lib.SIGNATURES.update(_SIGS)


def _fn(name):
    f = getattr(_lib.lib(), name)
    f.restype, f.argtypes = _SIGS[name]
    return f


def _call(name, *args):
    _lib.check(_fn(name)(*args), name)


@dataclass
class InstanceSpec:
    model: DiffusionModel
    lam: List[float]
    seed: int
    realisation: int = 0
    max_snapshots: int = 0
    flags: int = 0


class Ensemble:
    def __init__(self, specs: List[InstanceSpec]):
        n = len(specs)
        inst = (Instance * n)()
        diff, lam, reac = [], [], []
        off = 0
        snap_off = 0
        self.offsets = []
        self.snap_offsets = []
        self.shapes = []
        for i, sp in enumerate(specs):
            m = sp.model
            if m.width != m.height:
                raise ValueError("ensemble instances are square")
            I = inst[i]
            I.width = m.width
            I.num_species = m.num_species
            I.num_reactions = len(m.reactions)
            I.species_offset = len(diff)
            I.reaction_offset = len(reac)
            for k in range(4):
                I.boundary_mask[k] = int(m.boundary_mask[k])
            I.physical_length, I.p0 = m.physical_length, m.p0
            I.max_time, I.output_interval = m.max_time, m.output_interval
            I.max_steps = m.max_steps
            I.flags = sp.flags | m.flags
            I.seed, I.realisation = sp.seed & 0xFFFFFFFF, sp.realisation
            I.max_snapshots = sp.max_snapshots
            I.state_offset = off
            block = m.num_species * m.area
            if sp.max_snapshots > 0:
                I.snapshot_offset = snap_off
                self.snap_offsets.append(snap_off)
                snap_off += sp.max_snapshots * block
            else:
                I.snapshot_offset = -1
                self.snap_offsets.append(-1)
            self.offsets.append(off)
            self.shapes.append((m.num_species, m.height, m.width))
            off += block
            diff += [s.diffusion for s in m.species]
            lam += list(sp.lam)
            arr = m.reaction_array()
            reac += [arr[k] for k in range(len(m.reactions))]
        self.n = n
        self.state_size = off
        self.snap_size = snap_off
        self.specs = specs
        self._diff = np.asarray(diff, np.float32)
        self._lam = np.asarray(lam, np.float32)
        nr = max(1, len(reac))
        self._reac = (_lib.Reaction * nr)(*reac) if reac else (_lib.Reaction * 1)()
        self._inst = inst
        h = C.c_void_p()
        _call("gpgmp_ensemble_create", inst, n, self._diff.ctypes.data_as(P(f32)), len(diff),
              self._lam.ctypes.data_as(P(f32)), self._reac, len(reac), C.byref(h))
        self._h = h

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            _fn("gpgmp_ensemble_destroy")(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def alloc_state(self):
        import torch
        return torch.zeros(self.state_size, dtype=torch.int32, device="cuda")

    def alloc_snapshots(self):
        import torch
        return torch.zeros(max(1, self.snap_size), dtype=torch.int32, device="cuda")

    def configure(self, threads: int, ctas_per_sm: int):
        _call("gpgmp_ensemble_configure", self._h, threads, ctas_per_sm)

    def launch_shape(self):
        a, b, c = C.c_int32(), C.c_int32(), C.c_int32()
        _call("gpgmp_ensemble_launch_shape", self._h, C.byref(a), C.byref(b), C.byref(c))
        return a.value, b.value, c.value

    def init_poisson(self, state):
        import torch
        _call("gpgmp_ensemble_init_poisson", self._h, C.c_void_p(state.data_ptr()),
              C.c_void_p(torch.cuda.current_stream().cuda_stream))

    def run(self, state, snapshots=None):
        import torch
        _call("gpgmp_ensemble_run", self._h, C.c_void_p(state.data_ptr()),
              C.c_void_p(snapshots.data_ptr()) if snapshots is not None else None,
              C.c_void_p(torch.cuda.current_stream().cuda_stream))

    def results(self):
        st = np.zeros(self.n, np.int32)
        steps = np.zeros(self.n, np.int64)
        nt = sum(max(0, s.max_snapshots) for s in self.specs)
        times = np.zeros(max(1, nt), np.float32)
        _call("gpgmp_ensemble_results", self._h, st.ctypes.data_as(P(i32)), steps.ctypes.data_as(P(i64)),
              times.ctypes.data_as(P(f32)))
        return st, steps, times[:nt]

    def instance_state(self, state, i):
        S, H, W = self.shapes[i]
        o = self.offsets[i]
        return state[o:o + S * H * W].view(S, H, W)

    def cell_steps(self, steps: np.ndarray) -> int:
        return int(sum(H * W * int(s) for (S, H, W), s in zip(self.shapes, steps)))


# ---------------------------------------------------------------------------------
# Workloads
# ---------------------------------------------------------------------------------

def replicate(model: DiffusionModel, lam, R: int, seed: int, max_snapshots: int = 0) -> List[InstanceSpec]:
    """R realisations of one model; realisation r has the stream key (seed, r), as in
    a gpgmp_solver of R realisations."""
    return [InstanceSpec(model, list(lam), seed, r, max_snapshots) for r in range(R)]


def random_instance(rng: np.random.Generator, max_time: float = 5.0) -> (DiffusionModel, List[float]):
    """One random instance of the heterogeneous ensemble: side ~ U{16..128},
    species ~ U{4..12}, reactions ~ U{8..32} of order ~ U{0,1,2} (reactants drawn
    uniformly with replacement) with 0-2 product molecules (uniform species),
    rates log-uniform in [1e-3, 1], D ~ U[0.1, 2], initial counts Poisson(lambda)
    with lambda ~ U[10, 200]; h = 1, p0 = 0.1, reflecting walls; one output at the end
    time; a count that would pass INT32_MAX stops the instance with a status bit."""
    side = int(rng.integers(16, 129))
    S = int(rng.integers(4, 13))
    R = int(rng.integers(8, 33))
    m = DiffusionModel(width=side, height=side, physical_length=float(side), p0=0.1, max_time=max_time,
                       output_interval=max_time, flags=_lib.FLAG_STOP_ON_ERROR)
    names = [f"S{k}" for k in range(S)]
    for nm in names:
        m.add_species(nm, float(rng.uniform(0.1, 2.0)))
    for r in range(R):
        order = int(rng.integers(0, 3))
        reac = {}
        for _ in range(order):
            nm = names[int(rng.integers(0, S))]
            reac[nm] = reac.get(nm, 0) + 1
        prod = {}
        for _ in range(int(rng.integers(0, 3))):
            nm = names[int(rng.integers(0, S))]
            prod[nm] = prod.get(nm, 0) + 1
        rate = float(10.0 ** rng.uniform(-3.0, 0.0))
        m.add_reaction(f"r{r}", reac, prod, rate)
    lam = [float(rng.uniform(10.0, 200.0)) for _ in range(S)]
    return m, lam


def random_ensemble(n: int, seed: int, max_time: float = 5.0) -> List[InstanceSpec]:
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for i in range(n):
        m, lam = random_instance(rng, max_time)
        out.append(InstanceSpec(m, lam, seed=(seed * 7919 + i) & 0xFFFFFFFF, realisation=0))
    return out


# ---------------------------------------------------------------------------------
# Autotuner: launch shape of the persistent kernel
# ---------------------------------------------------------------------------------

TUNE_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_tune")
CANDIDATES = [(256, 2), (256, 4), (512, 1), (512, 2), (1024, 1)]


def _signature(specs: List[InstanceSpec]) -> str:
    sides = np.array([s.model.width for s in specs])
    S = np.array([s.model.num_species for s in specs])
    R = np.array([len(s.model.reactions) for s in specs])
    return f"n{len(specs)}_w{int(sides.mean())}_{int(sides.max())}_s{int(S.mean())}_r{int(R.mean())}"


def autotune(specs: List[InstanceSpec], sample: int = 256, seed: int = 0, cache: bool = True):
    """Times every candidate (threads per CTA, CTAs per SM) on a sample of the
    instances (shortened to a tenth of their end time) and returns the fastest;
    results are cached per GPU and workload signature under inchman_b200/_tune/."""
    import torch
    name = torch.cuda.get_device_name().replace(" ", "_")
    key = f"{name}_{_signature(specs)}"
    path = os.path.join(TUNE_DIR, key + ".json")
    if cache and os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return tuple(d["best"]), d
    rng = np.random.default_rng(seed)
    pick = rng.choice(len(specs), size=min(sample, len(specs)), replace=False)
    sub = []
    for i in pick:
        s = specs[int(i)]
        m = DiffusionModel(**{k: getattr(s.model, k) for k in ("width", "height", "physical_length", "p0",
                                                                 "output_interval", "max_steps", "boundary_mask",
                                                                 "source_mask", "solver", "flags")})
        m.species, m.reactions = s.model.species, s.model.reactions
        m.max_time = s.model.max_time / 10.0
        m.output_interval = m.max_time
        sub.append(InstanceSpec(m, s.lam, s.seed, s.realisation))
    ens = Ensemble(sub)
    state = ens.alloc_state()
    timings = {}
    for thr, cps in CANDIDATES:
        try:
            ens.configure(thr, cps)
        except _lib.GpgmpError:
            continue
        ens.init_poisson(state)
        ens.run(state)
        torch.cuda.synchronize()
        ens.init_poisson(state)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        ens.run(state)
        b.record()
        torch.cuda.synchronize()
        timings[f"{thr}x{cps}"] = a.elapsed_time(b)
    best = min(timings, key=timings.get)
    thr, cps = (int(v) for v in best.split("x"))
    d = {"best": [thr, cps], "ms": timings, "sample": len(sub)}
    if cache:
        os.makedirs(TUNE_DIR, exist_ok=True)
        with open(path, "w") as f:
            json.dump(d, f, indent=1)
    return (thr, cps), d


def main(argv=None):
    """Runs a random heterogeneous ensemble (the batched workload's generator) twice
    and prints the time and cell-steps/s of each run:
        python -m inchman_b200.ensemble [--instances N] [--max-time T] [--threads K]"""
    import argparse
    import torch
    ap = argparse.ArgumentParser()
    ap.add_argument("--instances", type=int, default=296)
    ap.add_argument("--max-time", type=float, default=0.5)
    ap.add_argument("--threads", type=int, default=1024)
    ap.add_argument("--ctas-per-sm", type=int, default=1)
    ap.add_argument("--seed", type=int, default=2024)
    a = ap.parse_args(argv)
    ens = Ensemble(random_ensemble(a.instances, seed=a.seed, max_time=a.max_time))
    ens.configure(a.threads, a.ctas_per_sm)
    state = ens.alloc_state()
    for k in range(2):
        ens.init_poisson(state)
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record()
        ens.run(state)
        t1.record()
        torch.cuda.synchronize()
        status, steps, _ = ens.results()
        ms = t0.elapsed_time(t1)
        print(f"run {k}: {ms:.1f} ms, {ens.cell_steps(steps) / ms * 1e3:.3e} cell-steps/s, "
              f"{int((status != 0).sum())} instances with status bits")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
