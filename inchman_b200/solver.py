"""Python mirror of the reference's solver interface over the C ABI.

    s = Solver(model, realisations=16, seed=1234)
    s.init_poisson([100, 100, 0])
    s.do_reactions(dt, seed)            # Solver::doReactions      (Solver.h:52)
    s.diffuse(i, t, seed)               # Solver::diffuse          (Solver.h:80)
    s.get_next_diffusion_time()         # Solver::getNextDiffusionTime (Solver.h:68)
    s.synchronize_state_from_device()   # Solver::synchronizeStateBufferFromDevice (Solver.h:85)
    s.solve()                           # DiffusionModel::oclSolve (DiffusionModel.cpp:1414)

HomogeneousSolver / InhomogeneousSolver are the same class chosen by the
model's solver type, as oclSolve picks them (DiffusionModel.cpp:1425-1440).
"""
from __future__ import annotations

import ctypes as C
import json
import os
from typing import Optional, Sequence

import numpy as np

from . import _lib
from .model import DiffusionModel


TUNE_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_tune")


def _device_name() -> str:
    try:
        import torch
        return torch.cuda.get_device_name().replace(" ", "_")
    except Exception:
        return "gpu"


class Solver:
    def __init__(self, model: DiffusionModel, realisations: int = 1, seed: int = 0, sync_each_launch: bool = False,
                 stream: Optional[int] = None):
        self.model = model
        self.R = int(realisations)
        self.seed = int(seed) & 0xFFFFFFFF
        self._desc, self._keep = model.to_desc()
        h = C.c_void_p()
        flags = _lib.CREATE_SYNC_EACH_LAUNCH if sync_each_launch else 0
        _lib.call("gpgmp_solver_create", C.byref(self._desc), self.R, self.seed, flags, C.byref(h))
        self._h = h
        self.deterministic = model.solver in _lib.DETERMINISTIC_TYPES
        self.dtype = np.float32 if self.deterministic else np.int32
        if stream is not None:
            _lib.call("gpgmp_solver_set_stream", self._h, C.c_void_p(stream))

    @property
    def shape(self):
        m = self.model
        return (self.R, m.num_species, m.height, m.width)

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            _lib.lib().gpgmp_solver_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- launch shapes ----------------------------------------------------------
    @staticmethod
    def launch_choices():
        """([(tile_w, tile_h), ...], [ssa_threads, ...]): the shapes the kernels can run."""
        nt, ns = C.c_int32(), C.c_int32()
        tw, th, st = (C.c_int32 * 8)(), (C.c_int32 * 8)(), (C.c_int32 * 8)()
        _lib.call("gpgmp_solver_launch_choices", C.byref(nt), tw, th, C.byref(ns), st)
        return [(tw[i], th[i]) for i in range(nt.value)], [st[i] for i in range(ns.value)]

    def set_launch(self, tile=(32, 16), ssa_threads: int = 128):
        _lib.call("gpgmp_solver_set_launch", self._h, int(tile[0]), int(tile[1]), int(ssa_threads))

    def get_launch(self):
        w, h, t = C.c_int32(), C.c_int32(), C.c_int32()
        _lib.call("gpgmp_solver_get_launch", self._h, C.byref(w), C.byref(h), C.byref(t))
        return (w.value, h.value), t.value

    def autotune(self, window: float = 0.0, reps: int = 3, cache: bool = True):
        """Picks the fastest diffusion tile shape and SSA block size for this solver's
        model on the current state (gpgmp_solver_autotune) and returns
        {"tile": (w, h), "ssa_threads": n, "ms_tiles": {...}, "ms_ssa": {...}}.  The choice
        is cached per GPU and workload signature (grid, realisations, species,
        reactions, solver type) under inchman_b200/_tune/ and taken from there next
        time; the results do not depend on it."""
        tiles, ssas = self.launch_choices()
        m = self.model
        key = f"solver_{_device_name()}_{m.solver}_{m.width}x{m.height}_R{self.R}_S{m.num_species}" \
              f"_N{len(m.reactions)}{'_masked' if m.reaction_mask() is not None else ''}"
        path = os.path.join(TUNE_DIR, key + ".json")
        if cache and os.path.exists(path):
            with open(path) as f:
                d = json.load(f)
            self.set_launch(tuple(d["tile"]), d["ssa_threads"])
            return d
        mt, ms = (C.c_float * len(tiles))(), (C.c_float * len(ssas))()
        _lib.call("gpgmp_solver_autotune", self._h, float(window), int(reps), mt, ms)
        tile, thr = self.get_launch()
        d = {"tile": list(tile), "ssa_threads": thr,
             "ms_tiles": {f"{w}x{h}": mt[i] for i, (w, h) in enumerate(tiles)},
             "ms_ssa": {str(t): ms[i] for i, t in enumerate(ssas)}}
        if cache:
            os.makedirs(TUNE_DIR, exist_ok=True)
            with open(path, "w") as f:
                json.dump(d, f, indent=1)
        return d

    # -- state --------------------------------------------------------------------
    def set_state(self, state: np.ndarray):
        a = np.ascontiguousarray(state, dtype=self.dtype)
        if a.size != int(np.prod(self.shape)):
            raise ValueError(f"state must hold {self.shape} values")
        _lib.call("gpgmp_set_state", self._h, a.ctypes.data_as(C.c_void_p))

    synchronize_state_to_device = set_state

    def get_state(self) -> np.ndarray:
        out = np.empty(self.shape, dtype=self.dtype)
        _lib.call("gpgmp_get_state", self._h, out.ctypes.data_as(C.c_void_p))
        return out

    synchronize_state_from_device = get_state

    def init_poisson(self, lam: Sequence[float]):
        a = np.ascontiguousarray(lam, dtype=np.float32)
        _lib.call("gpgmp_init_poisson", self._h, a.ctypes.data_as(C.POINTER(C.c_float)))

    def device_state_ptr(self) -> int:
        return _lib.lib().gpgmp_device_state(self._h) or 0

    # -- the Solver virtuals ---------------------------------------------------------
    def do_reactions(self, deltat: float, seed: int) -> int:
        s = C.c_int32(seed)
        _lib.call("gpgmp_do_reactions", self._h, C.c_float(deltat), C.byref(s))
        return s.value

    def diffuse(self, species: int, current_time: float, seed: int) -> int:
        s = C.c_int32(seed)
        _lib.call("gpgmp_diffuse", self._h, int(species), C.c_float(current_time), C.byref(s))
        return s.value

    def get_next_diffusion_time(self) -> np.ndarray:
        out = np.empty(self.model.num_species, dtype=np.float32)
        _lib.call("gpgmp_next_diffusion_time", self._h, out.ctypes.data_as(C.POINTER(C.c_float)))
        return out

    def timesteps(self):
        S = self.model.num_species
        dx = np.empty(S, dtype=np.float32)
        dy = np.empty(S, dtype=np.float32)
        _lib.call("gpgmp_timesteps", self._h, dx.ctypes.data_as(C.POINTER(C.c_float)),
                  dy.ctypes.data_as(C.POINTER(C.c_float)))
        return dx, dy

    # -- field parameters ------------------------------------------------------------
    def get_fields(self) -> np.ndarray:
        """The field parameters [F][H][W] (synchronizeFieldBufferFromDevice)."""
        m = self.model
        out = np.zeros((len(m.field_names), m.height, m.width), np.float32)
        if out.size:
            _lib.call("gpgmp_get_fields", self._h, out.ctypes.data_as(C.POINTER(C.c_float)))
        return out

    def set_fields(self, fields):
        a = np.ascontiguousarray(fields, dtype=np.float32)
        _lib.call("gpgmp_set_fields", self._h, a.ctypes.data_as(C.POINTER(C.c_float)))

    def update_fields(self, deltat: float, simtime: float):
        """One pass of the setField method (Solver::updateFields)."""
        _lib.call("gpgmp_update_fields", self._h, C.c_float(deltat), C.c_float(simtime))

    # -- individual species (IndividualSolver) --------------------------------------
    def individual_count(self, species: int) -> int:
        n = C.c_int64(0)
        _lib.call("gpgmp_individual_count", self._h, int(species), C.byref(n))
        return n.value

    def get_individuals(self, species: int):
        """(keys, ids, props): keys r * area + cell in list order (sorted), ids, and
        props [4][n] = DiffusivityX, DiffusivityY, DriftX, DriftY."""
        n = self.individual_count(species)
        keys = np.empty(n, np.uint32)
        ids = np.empty(n, np.uint32)
        props = np.empty((4, n), np.float32)
        got = C.c_int64(0)
        _lib.call("gpgmp_get_individuals", self._h, int(species), keys.ctypes.data_as(C.c_void_p),
                  ids.ctypes.data_as(C.c_void_p), props.ctypes.data_as(C.c_void_p), n, C.byref(got))
        return keys, ids, props

    def set_individual_properties(self, species: int, props, first_id: int = 0):
        """props [4][count] for ids first_id ..: DiffusivityX, DiffusivityY, DriftX, DriftY
        (what the reference's init scripts set through individualProperties)."""
        a = np.ascontiguousarray(props, dtype=np.float32)
        if a.ndim != 2 or a.shape[0] != 4:
            raise ValueError("props must be [4][count]")
        _lib.call("gpgmp_set_individual_properties", self._h, int(species), a.ctypes.data_as(C.c_void_p),
                  int(first_id), a.shape[1])

    def status(self) -> np.ndarray:
        out = np.zeros(self.R, dtype=np.int32)
        _lib.call("gpgmp_get_status", self._h, out.ctypes.data_as(C.POINTER(C.c_int32)))
        return out

    def synchronize(self):
        _lib.call("gpgmp_synchronize", self._h)

    def solve(self, max_snapshots: int = 0, count_only: bool = False, on_dump=None):
        """Runs the oclSolve event loop; returns (snapshots, times, steps).  on_dump(index,
        time) is called at every dump, when the solver's state and individual lists are
        those of the dump (the reference's writeAllSpecies)."""
        if on_dump is not None:
            snaps = np.zeros((max(1, max_snapshots),) + self.shape, dtype=self.dtype)
            times = np.zeros(max(1, max_snapshots), dtype=np.float32)
            ns = C.c_int32(0)
            steps = C.c_int64(0)
            errors = []

            def cb(_user, index, t):
                try:
                    on_dump(int(index), float(t))
                    return 0
                except Exception as e:       # reported after the run
                    errors.append(e)
                    return 1

            fn = _lib.DUMP_CALLBACK(cb)
            try:
                _lib.call("gpgmp_solve_with_callback", self._h, snaps.ctypes.data_as(C.c_void_p),
                          times.ctypes.data_as(C.POINTER(C.c_float)), max_snapshots, C.byref(ns), C.byref(steps),
                          C.cast(fn, C.c_void_p), None)
            except _lib.GpgmpError:
                if errors:
                    raise errors[0]
                raise
            n = min(ns.value, max_snapshots)
            return snaps[:n], times[:n], steps.value
        if count_only or max_snapshots == 0:
            ns = C.c_int32(0)
            steps = C.c_int64(0)
            _lib.call("gpgmp_solve", self._h, None, None, 0, C.byref(ns), C.byref(steps))
            return None, None, steps.value
        snaps = np.zeros((max_snapshots,) + self.shape, dtype=self.dtype)
        times = np.zeros(max_snapshots, dtype=np.float32)
        ns = C.c_int32(0)
        steps = C.c_int64(0)
        _lib.call("gpgmp_solve", self._h, snaps.ctypes.data_as(C.c_void_p),
                  times.ctypes.data_as(C.POINTER(C.c_float)), max_snapshots, C.byref(ns), C.byref(steps))
        n = min(ns.value, max_snapshots)
        return snaps[:n], times[:n], steps.value


HomogeneousSolver = Solver
InhomogeneousSolver = Solver
