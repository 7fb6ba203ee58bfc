"""Individual-particle path: exclusive scan, radix sort, cell offsets and the
particle binning step, over the C ABI.

Device-pointer primitives take torch CUDA tensors (uint32 values travel as int32
tensors of the same bits):
    exclusive_scan_u32(x)            -> out[i] = x[0] + ... + x[i-1] (mod 2^32)
    sort_pairs_u32(keys, vals, bits) -> stable sort by the low `bits` key bits
    cell_offsets(sorted_keys, ncells) -> (start, count)
    cell_indices(start, count)        -> the reference's (left, right) ranges
    maintain_population(...)          -> the individual list brought to new counts
Particles(capacity, grid, ...) wraps the move/bin/react/compact step.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib

vp, i32, i64, u32, f32 = C.c_void_p, C.c_int32, C.c_int64, C.c_uint32, C.c_float
P = C.POINTER

_SIGS = {
    "gpgmp_scan_scratch_bytes": (C.c_int, [i64, P(C.c_size_t)]),
    "gpgmp_exclusive_scan_u32": (C.c_int, [vp, vp, i64, vp, C.c_size_t, vp]),
    "gpgmp_sort_scratch_bytes": (C.c_int, [i64, i32, P(C.c_size_t)]),
    "gpgmp_sort_pairs_u32": (C.c_int, [vp, vp, vp, vp, i64, i32, vp, C.c_size_t, vp]),
    "gpgmp_cell_offsets": (C.c_int, [vp, i64, i64, vp, vp, vp, C.c_size_t, vp]),
    "gpgmp_cell_indices": (C.c_int, [vp, vp, i64, vp, vp, vp]),
    "gpgmp_scratch_status": (C.c_int, [vp, i32, i64, i32, P(i32)]),
    "gpgmp_population_scratch_bytes": (C.c_int, [i64, i64, P(C.c_size_t)]),
    "gpgmp_population_maintain": (C.c_int, [vp, vp, i64, vp, vp, vp, i64, vp, i64, u32, u32, vp, vp, i64, vp, i64,
                                            vp, P(i64), P(i64), vp, C.c_size_t, vp]),
    "gpgmp_particles_create": (C.c_int, [i64, i32, f32, f32, f32, f32, f32, u32, P(vp)]),
    "gpgmp_particles_destroy": (C.c_int, [vp]),
    "gpgmp_particles_set_stream": (C.c_int, [vp, vp]),
    "gpgmp_particles_set": (C.c_int, [vp, vp, vp, vp, i64, i32]),
    "gpgmp_particles_get": (C.c_int, [vp, vp, vp, vp, P(i64)]),
    "gpgmp_particles_step": (C.c_int, [vp, i32]),
    "gpgmp_particles_bins": (C.c_int, [vp, vp, vp, vp, vp, P(i64)]),
    "gpgmp_particles_status": (C.c_int, [vp, P(i32)]),
}
_lib.SIGNATURES.update(_SIGS)


def _fn(name):
    f = getattr(_lib.lib(), name)
    f.restype, f.argtypes = _SIGS[name]
    return f


def _call(name, *args):
    _lib.check(_fn(name)(*args), name)


def _stream():
    import torch
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def scan_scratch(n: int, device="cuda"):
    import torch
    b = C.c_size_t(0)
    _call("gpgmp_scan_scratch_bytes", n, C.byref(b))
    return torch.empty(max(1, b.value), dtype=torch.uint8, device=device)


def exclusive_scan_u32(x, scratch=None):
    """x: int32/uint32-bit CUDA tensor; returns the exclusive prefix sums mod 2^32."""
    import torch
    x = x.contiguous()
    out = torch.empty_like(x)
    n = x.numel()
    if scratch is None:
        scratch = scan_scratch(n, x.device)
    _call("gpgmp_exclusive_scan_u32", _ptr(x), _ptr(out), n, _ptr(scratch), scratch.numel(), _stream())
    return out


def sort_scratch(n: int, key_bits: int, device="cuda"):
    import torch
    b = C.c_size_t(0)
    _call("gpgmp_sort_scratch_bytes", n, key_bits, C.byref(b))
    return torch.empty(max(1, b.value), dtype=torch.uint8, device=device)


def sort_pairs_u32(keys, vals, key_bits: int = 32, scratch=None):
    import torch
    keys = keys.contiguous()
    vals = vals.contiguous()
    n = keys.numel()
    ko = torch.empty_like(keys)
    vo = torch.empty_like(vals)
    if scratch is None:
        scratch = sort_scratch(n, key_bits, keys.device)
    _call("gpgmp_sort_pairs_u32", _ptr(keys), _ptr(vals), _ptr(ko), _ptr(vo), n, key_bits, _ptr(scratch),
          scratch.numel(), _stream())
    return ko, vo, scratch


def scratch_status(scratch, kind: int, n: int = 0, key_bits: int = 32) -> int:
    st = C.c_int32(0)
    _call("gpgmp_scratch_status", _ptr(scratch), kind, n, key_bits, C.byref(st))
    return st.value


def cell_offsets(sorted_keys, ncells: int, scratch=None):
    import torch
    start = torch.empty(ncells, dtype=torch.int32, device=sorted_keys.device)
    count = torch.empty(ncells, dtype=torch.int32, device=sorted_keys.device)
    if scratch is None:
        scratch = scan_scratch(ncells, sorted_keys.device)
    _call("gpgmp_cell_offsets", _ptr(sorted_keys), sorted_keys.numel(), ncells, _ptr(start), _ptr(count),
          _ptr(scratch), scratch.numel(), _stream())
    return start, count


def cell_indices(start, count):
    import torch
    left = torch.empty_like(start)
    right = torch.empty_like(start)
    _call("gpgmp_cell_indices", _ptr(start), _ptr(count), start.numel(), _ptr(left), _ptr(right), _stream())
    return left, right


def maintain_population(keys, ids, start, count, goal, pool, seed: int, step: int, capacity: int = None,
                        pool_capacity: int = None):
    """IndividualSolver::maintainPopulation: rebuild the cell-sorted individual list
    (keys = cell, ids, with start / count from cell_offsets) so that cell c holds
    goal[c] individuals.  Returns (keys, ids, start, pool) of the new list and pool
    (int32 tensors of uint32 bits; counts are goal)."""
    import torch
    dev = goal.device
    n, ncells, npool = keys.numel(), goal.numel(), pool.numel()
    cap = capacity if capacity is not None else n + npool
    pcap = pool_capacity if pool_capacity is not None else n + npool
    b = C.c_size_t(0)
    _call("gpgmp_population_scratch_bytes", n, ncells, C.byref(b))
    scratch = torch.empty(max(1, b.value), dtype=torch.uint8, device=dev)
    ko = torch.empty(max(1, cap), dtype=torch.int32, device=dev)
    io = torch.empty_like(ko)
    po = torch.empty(max(1, pcap), dtype=torch.int32, device=dev)
    so = torch.empty(ncells, dtype=torch.int32, device=dev)
    na, npo = C.c_int64(0), C.c_int64(0)
    _call("gpgmp_population_maintain", _ptr(keys) if n else None, _ptr(ids) if n else None, n, _ptr(start),
          _ptr(count), _ptr(goal), ncells, _ptr(pool) if npool else None, npool, seed & 0xFFFFFFFF,
          step & 0xFFFFFFFF, _ptr(ko), _ptr(io), cap, _ptr(po), pcap, _ptr(so), C.byref(na), C.byref(npo),
          _ptr(scratch), scratch.numel(), _stream())
    return ko[:na.value], io[:na.value], so, po[:npo.value]


class Particles:
    """2-D lattice particles (positions, species A=0 / B=1) with the binning step."""

    def __init__(self, capacity: int, grid: int, D: float, vx: float, vy: float, dt: float, p_react: float,
                 seed: int):
        h = C.c_void_p()
        _call("gpgmp_particles_create", capacity, grid, D, vx, vy, dt, p_react, seed & 0xFFFFFFFF, C.byref(h))
        self._h = h
        self.grid = grid

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            _fn("gpgmp_particles_destroy")(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set(self, x, y, species, step: int = 0):
        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.ascontiguousarray(y, dtype=np.float32)
        sp = np.ascontiguousarray(species, dtype=np.uint8)
        _call("gpgmp_particles_set", self._h, x.ctypes.data_as(vp), y.ctypes.data_as(vp), sp.ctypes.data_as(vp),
              x.size, step)

    def get(self):
        n = C.c_int64(0)
        _call("gpgmp_particles_get", self._h, None, None, None, C.byref(n))
        x = np.empty(n.value, np.float32)
        y = np.empty(n.value, np.float32)
        sp = np.empty(n.value, np.uint8)
        _call("gpgmp_particles_get", self._h, x.ctypes.data_as(vp), y.ctypes.data_as(vp), sp.ctypes.data_as(vp),
              C.byref(n))
        return x, y, sp

    def step(self, n: int = 1):
        _call("gpgmp_particles_step", self._h, n)

    def bins(self):
        nc = self.grid * self.grid
        start = np.empty(nc, np.uint32)
        count = np.empty(nc, np.uint32)
        nb = C.c_int64(0)
        _call("gpgmp_particles_bins", self._h, start.ctypes.data_as(vp), count.ctypes.data_as(vp), None, None,
              C.byref(nb))
        keys = np.empty(nb.value, np.uint32)
        idx = np.empty(nb.value, np.uint32)
        _call("gpgmp_particles_bins", self._h, start.ctypes.data_as(vp), count.ctypes.data_as(vp),
              keys.ctypes.data_as(vp), idx.ctypes.data_as(vp), C.byref(nb))
        return start, count, keys, idx

    def status(self) -> int:
        st = C.c_int32(0)
        _call("gpgmp_particles_status", self._h, C.byref(st))
        return st.value


def uniform_particles(n: int, grid: int, seed: int):
    """Seeded uniform initial positions in [0, grid)^2 and species A/B half each."""
    rng = np.random.Generator(np.random.PCG64(seed))
    x = rng.uniform(0.0, grid, size=n).astype(np.float32)
    y = rng.uniform(0.0, grid, size=n).astype(np.float32)
    x = np.minimum(x, np.nextafter(np.float32(grid), np.float32(0)))
    y = np.minimum(y, np.nextafter(np.float32(grid), np.float32(0)))
    sp = (np.arange(n) % 2).astype(np.uint8)
    rng.shuffle(sp)
    return x, y, sp
