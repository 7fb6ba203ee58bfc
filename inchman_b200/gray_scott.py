"""Deterministic Gray-Scott reaction-diffusion on the GPU, forward and adjoint.

The reference's deterministic solver (exec/src/gpgmp/src/Deterministic.cl:17-238)
on the Gray-Scott network (exec/src/tests/GrayScottModel.cpp:14-60), explicit Euler
steps on a periodic n x n lattice with an optional constant drift, computed by the
cluster-resident kernels of csrc/gray_scott.cu through the C ABI.

GrayScott.apply(u0, v0, theta) is a torch.autograd.Function: theta holds
(F, k, Du, Dv, vx, vy); backward runs the hand-written adjoint with two-level
checkpointing and returns gradients for u0, v0 and theta.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib

PARAM_NAMES = ("F", "k", "Du", "Dv", "vx", "vy")


class GSParams(C.Structure):
    _fields_ = [("n", C.c_int32), ("steps", C.c_int32),
                ("F", C.c_double), ("k", C.c_double), ("Du", C.c_double), ("Dv", C.c_double),
                ("vx", C.c_double), ("vy", C.c_double), ("dt", C.c_double),
                ("checkpoint_every", C.c_int32), ("cluster", C.c_int32), ("variant", C.c_int32)]


_SIGS = {
    "gpgmp_gs_buffer_sizes": (C.c_int, [C.POINTER(GSParams), C.c_int32, C.POINTER(C.c_size_t),
                                        C.POINTER(C.c_size_t)]),
    "gpgmp_gs_forward_f32": (C.c_int, [C.POINTER(GSParams)] + [C.c_void_p] * 6),
    "gpgmp_gs_forward_f64": (C.c_int, [C.POINTER(GSParams)] + [C.c_void_p] * 6),
    "gpgmp_gs_adjoint_f32": (C.c_int, [C.POINTER(GSParams)] + [C.c_void_p] * 8),
    "gpgmp_gs_adjoint_f64": (C.c_int, [C.POINTER(GSParams)] + [C.c_void_p] * 8),
    "gpgmp_gs_forward_host": (C.c_int, [C.POINTER(GSParams)] + [C.c_void_p] * 4),
    "gpgmp_gs_loss_grad_host": (C.c_int, [C.POINTER(GSParams)] + [C.c_void_p] * 6),
    "gpgmp_gs_status": (C.c_int, [C.POINTER(C.c_int32)]),
    "gpgmp_gs_forward_batch_f32": (C.c_int, [C.POINTER(GSParams), C.c_int32, C.c_void_p] + [C.c_void_p] * 5),
    "gpgmp_gs_batch_capacity": (C.c_int, [C.c_int32, C.POINTER(C.c_int32)]),
    "gpgmp_gs_auto_variant": (C.c_int, [C.c_int32, C.c_int32, C.POINTER(C.c_int32)]),
}
_lib.SIGNATURES.update(_SIGS)


def _fn(name):
    L = _lib.lib()
    f = getattr(L, name)
    res, args = _SIGS[name]
    f.restype, f.argtypes = res, args
    return f


@dataclass
class GrayScottConfig:
    """The Gray-Scott workload: 256 x 256 periodic, F=0.04, k=0.06, Du=0.16, Dv=0.08,
    dt=1, 10,000 steps; u=1, v=0 with a central 20 x 20 square u=0.5, v=0.25, plus
    uniform(-0.01, 0.01) noise on both; target = the same run with F=0.042."""
    n: int = 256
    steps: int = 10_000
    F: float = 0.04
    k: float = 0.06
    Du: float = 0.16
    Dv: float = 0.08
    vx: float = 0.0
    vy: float = 0.0
    dt: float = 1.0
    checkpoint_every: int = 100
    cluster: int = 0
    variant: int = 0
    seed: int = 1234

    def params(self, **over) -> GSParams:
        d = dict(n=self.n, steps=self.steps, F=self.F, k=self.k, Du=self.Du, Dv=self.Dv, vx=self.vx, vy=self.vy,
                 dt=self.dt, checkpoint_every=self.checkpoint_every, cluster=self.cluster, variant=self.variant)
        d.update(over)
        p = GSParams()
        for k_, v_ in d.items():
            setattr(p, k_, v_)
        return p

    def theta(self):
        return [self.F, self.k, self.Du, self.Dv, self.vx, self.vy]

    def initial_state(self, dtype=np.float32):
        n = self.n
        u = np.ones((n, n), dtype=np.float64)
        v = np.zeros((n, n), dtype=np.float64)
        c0 = n // 2 - 10
        u[c0:c0 + 20, c0:c0 + 20] = 0.5
        v[c0:c0 + 20, c0:c0 + 20] = 0.25
        rng = np.random.Generator(np.random.PCG64(self.seed))
        u += rng.uniform(-0.01, 0.01, size=(n, n))
        v += rng.uniform(-0.01, 0.01, size=(n, n))
        return u.astype(dtype), v.astype(dtype)


def buffer_sizes(p: GSParams, elem_bytes: int):
    a, b = C.c_size_t(0), C.c_size_t(0)
    _lib.check(_fn("gpgmp_gs_buffer_sizes")(C.byref(p), elem_bytes, C.byref(a), C.byref(b)),
               "gpgmp_gs_buffer_sizes")
    return a.value, b.value


def _stream_ptr(torch, device):
    return C.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def forward(u0, v0, p: GSParams, checkpoints=None):
    """Device forward solve on torch tensors (float32 or float64)."""
    import torch
    u0 = u0.contiguous()
    v0 = v0.contiguous()
    u = torch.empty_like(u0)
    v = torch.empty_like(v0)
    name = "gpgmp_gs_forward_f64" if u0.dtype == torch.float64 else "gpgmp_gs_forward_f32"
    ck = C.c_void_p(checkpoints.data_ptr()) if checkpoints is not None else None
    _lib.check(_fn(name)(C.byref(p), C.c_void_p(u0.data_ptr()), C.c_void_p(v0.data_ptr()), C.c_void_p(u.data_ptr()),
                         C.c_void_p(v.data_ptr()), ck, _stream_ptr(torch, u0.device)), name)
    return u, v


def forward_batch(u0, v0, p: GSParams, member_params=None):
    """Independent float32 lattices u0, v0 [batch][n][n] in one launch (one 16-CTA
    cluster each); member_params: optional [batch][6] (F, k, Du, Dv, vx, vy)."""
    import torch
    u0 = u0.contiguous()
    v0 = v0.contiguous()
    u = torch.empty_like(u0)
    v = torch.empty_like(v0)
    mp = None
    if member_params is not None:
        mp = np.ascontiguousarray(member_params, dtype=np.float64).reshape(-1, 6)
    _lib.check(_fn("gpgmp_gs_forward_batch_f32")(C.byref(p), u0.shape[0],
                                                 mp.ctypes.data_as(C.c_void_p) if mp is not None else None,
                                                 C.c_void_p(u0.data_ptr()), C.c_void_p(v0.data_ptr()),
                                                 C.c_void_p(u.data_ptr()), C.c_void_p(v.data_ptr()),
                                                 _stream_ptr(torch, u0.device)), "gpgmp_gs_forward_batch_f32")
    return u, v


def batch_capacity(n: int) -> int:
    """Lattices of side n that forward_batch runs at the same time on this GPU."""
    c = C.c_int32(0)
    _lib.check(_fn("gpgmp_gs_batch_capacity")(n, C.byref(c)), "gpgmp_gs_batch_capacity")
    return int(c.value)


# multi-cluster float32 forward families: variant -> (16-CTA clusters, ghost rows per band side)
MULTI_CLUSTER = {40: (2, 8), 41: (4, 8), 42: (4, 16), 43: (8, 8), 44: (8, 16), 45: (4, 32), 46: (2, 32)}


def auto_variant(n: int, drift: bool = False) -> int:
    """The float32 kernel family that variant 0 resolves to for an n x n lattice on
    this GPU (41: four 16-CTA clusters, 8 ghost rows; 10 + w: one cluster, w warps per CTA; 2: the
    shared-memory column walk; 1: one cell per iteration)."""
    v = C.c_int32(0)
    _lib.check(_fn("gpgmp_gs_auto_variant")(n, int(drift), C.byref(v)), "gpgmp_gs_auto_variant")
    return int(v.value)


def status() -> int:
    """Flags of the forward kernels since the last call (synchronises the device):
    non-zero if a bounded halo wait inside a register-resident forward solve gave up
    (that solve's output is NaN).  Clears the flags."""
    f = C.c_int32(0)
    _lib.check(_fn("gpgmp_gs_status")(C.byref(f)), "gpgmp_gs_status")
    return int(f.value)


def adjoint(p: GSParams, checkpoints, lam_u, lam_v):
    import torch
    dt = lam_u.dtype
    eb = 8 if dt == torch.float64 else 4
    _, wb = buffer_sizes(p, eb)
    work = torch.empty(wb // eb, dtype=dt, device=lam_u.device)
    gu = torch.empty_like(lam_u)
    gv = torch.empty_like(lam_v)
    g6 = torch.zeros(6, dtype=torch.float64, device=lam_u.device)
    name = "gpgmp_gs_adjoint_f64" if eb == 8 else "gpgmp_gs_adjoint_f32"
    _lib.check(_fn(name)(C.byref(p), C.c_void_p(checkpoints.data_ptr()), C.c_void_p(lam_u.contiguous().data_ptr()),
                         C.c_void_p(lam_v.contiguous().data_ptr()), C.c_void_p(gu.data_ptr()),
                         C.c_void_p(gv.data_ptr()), C.c_void_p(g6.data_ptr()), C.c_void_p(work.data_ptr()),
                         _stream_ptr(torch, lam_u.device)), name)
    # the work buffer's last 16 bytes hold the kernels' status word
    status = work.view(torch.uint8)[wb - 16: wb - 12].view(torch.int32)
    if int(status.item()) != 0:
        raise _lib.GpgmpError(5, name, "a bounded wait for a TMA copy in the adjoint gave up")
    return gu, gv, g6


def _make_autograd():
    import torch

    class GrayScott(torch.autograd.Function):
        """(u0, v0, theta) -> (u_N, v_N); theta = (F, k, Du, Dv, vx, vy); checkpoint_every
        <= 0: the library's automatic interval (100 steps in float32, 25 in float64)."""

        @staticmethod
        def forward(ctx, u0, v0, theta, steps: int, dt: float, checkpoint_every: int = 0):
            th = theta.detach().double().cpu().tolist()
            n = u0.shape[-1]
            p = GSParams(n=n, steps=steps, F=th[0], k=th[1], Du=th[2], Dv=th[3], vx=th[4], vy=th[5], dt=dt,
                         checkpoint_every=checkpoint_every, cluster=0, variant=0)
            eb = 8 if u0.dtype == torch.float64 else 4
            ckb, _ = buffer_sizes(p, eb)
            ck = torch.empty(ckb // eb, dtype=u0.dtype, device=u0.device)
            u, v = forward(u0, v0, p, checkpoints=ck)
            ctx.p = p
            ctx.theta_dtype = theta.dtype
            ctx.save_for_backward(ck)
            return u, v

        @staticmethod
        def backward(ctx, gu, gv):
            (ck,) = ctx.saved_tensors
            if gu is None:
                gu = torch.zeros_like(ck[: ctx.p.n * ctx.p.n].view(ctx.p.n, ctx.p.n))
            if gv is None:
                gv = torch.zeros_like(gu)
            gu0, gv0, g6 = adjoint(ctx.p, ck, gu.contiguous(), gv.contiguous())
            return gu0, gv0, g6.to(ctx.theta_dtype), None, None, None

    return GrayScott


_GS = None


def GrayScott():
    """The autograd Function class (built on first use so that importing this module
    does not import torch)."""
    global _GS
    if _GS is None:
        _GS = _make_autograd()
    return _GS


def forward_host(cfg: GrayScottConfig, u0: np.ndarray, v0: np.ndarray):
    """Host arrays in, host arrays out (copies inside the call)."""
    p = cfg.params()
    u0 = np.ascontiguousarray(u0, dtype=np.float32)
    v0 = np.ascontiguousarray(v0, dtype=np.float32)
    u = np.empty_like(u0)
    v = np.empty_like(v0)
    _lib.check(_fn("gpgmp_gs_forward_host")(C.byref(p), u0.ctypes.data_as(C.c_void_p), v0.ctypes.data_as(C.c_void_p),
                                            u.ctypes.data_as(C.c_void_p), v.ctypes.data_as(C.c_void_p)),
               "gpgmp_gs_forward_host")
    return u, v


def loss_grad_host(cfg: GrayScottConfig, u0, v0, ut, vt):
    p = cfg.params()
    arrs = [np.ascontiguousarray(a, dtype=np.float32) for a in (u0, v0, ut, vt)]
    loss = C.c_double(0)
    g = np.zeros(6, dtype=np.float64)
    _lib.check(_fn("gpgmp_gs_loss_grad_host")(C.byref(p), *[a.ctypes.data_as(C.c_void_p) for a in arrs],
                                              C.cast(C.byref(loss), C.c_void_p), g.ctypes.data_as(C.c_void_p)),
               "gpgmp_gs_loss_grad_host")
    return loss.value, g
