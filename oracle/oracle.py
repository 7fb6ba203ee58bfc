"""TEST INFRASTRUCTURE ONLY: ctypes access to the CPU oracle (oracle/_build/liboracle.so)
and to the reference checker (oracle/_ref/libgpgmp_ref.so, the reference's own kernel
sources compiled for the CPU).  Only tests/, the smoke check and bench.py's CPU
baseline import this module; the product never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "_build", "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libgpgmp_ref.so")

_orc = None
_ref = None

vp, i32, u32, f32, i64, f64 = C.c_void_p, C.c_int32, C.c_uint32, C.c_float, C.c_int64, C.c_double
P = C.POINTER


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def build_ref():
    subprocess.run(["make", "-s", "-C", HERE, "ref"], check=True)


def ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def orc():
    global _orc
    if _orc is None:
        if not os.path.exists(ORACLE_LIB):
            build()
        L = C.CDLL(ORACLE_LIB)
        sig = {
            "orc_threefry2x32_20": (None, [vp, vp, vp]),
            "orc_philox4x32_10": (None, [vp, vp, vp]),
            "orc_philox_fill": (None, [u32, u32, u32, u32, u32, vp, C.c_int]),
            "orc_logf_many": (None, [vp, vp, C.c_int]),
            "orc_expf_many": (None, [vp, vp, C.c_int]),
            "orc_sincos2pi_many": (None, [vp, vp, vp, C.c_int]),
            "orc_binomial_many": (None, [u32, u32, vp, vp, vp, C.c_int]),
            "orc_poisson_many": (None, [u32, u32, vp, vp, C.c_int]),
            "orc_ref_stay_probability": (f32, [vp]),
            "orc_ref_cell_width": (f32, [vp]),
            "orc_ref_homog_diffuse": (None, [vp, vp, C.c_int, i32, vp]),
            "orc_ref_source_boundary": (None, [vp, vp, C.c_int, i32, C.c_int, C.c_int]),
            "orc_ref_gillespie": (None, [vp, vp, i32, f32]),
            "orc_ref_inhomog_diffuse": (None, [vp, vp, C.c_int, i32, f32, C.c_int, vp, vp, vp, vp, vp]),
            "orc_ref_timestep": (f32, [vp, C.c_int, C.c_int, vp, vp, vp, vp, vp]),
            "orc_ref_det_diffuse": (None, [vp, vp, vp, f32, C.c_int]),
            "orc_ref_rk4": (None, [vp, vp, f32]),
            "orc_ref_solve": (C.c_int, [vp, vp, u32, vp, vp, C.c_int, P(C.c_int), P(i64)]),
            "orc_ref_solve_many": (None, [vp, vp, C.c_int, u32, vp]),
            "orc_ref_set_species_streams": (None, [C.c_int]),
            "orc_ref_solve_inhom": (C.c_int, [vp, vp, u32, vp, vp, vp, vp, vp, vp, C.c_int, P(C.c_int), P(i64)]),
            "orc_ref_solve_many_snaps": (None, [vp, vp, C.c_int, u32, vp, vp, vp, vp, C.c_int, vp]),
            "orc_rep_init_poisson": (None, [C.c_int, C.c_int, C.c_int, C.c_int, u32, vp, vp]),
            "orc_rep_ssa": (None, [vp, vp, C.c_int, u32, u32, f32, vp]),
            "orc_rep_homog_diffuse": (None, [vp, vp, C.c_int, u32, C.c_int, u32]),
            "orc_rep_inhomog_sweep": (None, [vp, vp, C.c_int, u32, C.c_int, C.c_int, u32, f32, vp, vp]),
            "orc_rep_timestep": (f32, [vp, C.c_int, C.c_int, vp, vp]),
            "orc_rep_ind_sweep": (C.c_int64, [vp, vp, C.c_int, C.c_uint32, C.c_int, C.c_int, f32, C.c_uint32, vp, vp,
                                              C.c_int64, vp, C.c_int64, vp]),
            "orc_rep_ind_sort": (C.c_int64, [vp, vp, C.c_int64, C.c_int64, vp, vp]),
            "orc_rep_timestep_cells": (f32, [vp, vp, C.c_int64, f32]),
            "orc_rep_diffusivity_drift": (None, [vp, C.c_int, vp, vp, vp, vp]),
            "orc_rep_solve": (C.c_int, [vp, vp, C.c_int, u32, vp, vp, C.c_int, P(C.c_int), P(i64), vp]),
            "orc_gs_forward_f32": (None, [C.c_int, C.c_int, f32, f32, f32, f32, f32, f32, f32, vp, vp]),
            "orc_gs_forward_f64": (None, [C.c_int, C.c_int, f64, f64, f64, f64, f64, f64, f64, vp, vp]),
            "orc_gs_loss_grad_f64": (f64, [C.c_int, C.c_int, f64, f64, f64, f64, f64, f64, f64, vp, vp, vp, vp,
                                           C.c_int, vp]),
            "orc_det_solve": (C.c_int, [vp, vp, vp, vp, C.c_int, P(C.c_int), P(i64)]),
            "orc_det_sweep": (None, [vp, vp, vp, C.c_int, C.c_int, f32, f32, vp, vp]),
            "orc_aqss_cell": (C.c_int, [vp, vp, f32, C.c_int]),
            "orc_aqss": (C.c_int, [vp, vp, f32, C.c_int]),
            "orc_set_custom_hazard": (None, [vp]),
            "orc_population_maintain": (C.c_int, [vp, vp, i64, vp, vp, vp, i64, vp, i64, u32, u32, vp, vp, vp,
                                                  P(i64), P(i64)]),
            "orc_sort_pairs_u32": (None, [vp, vp, i64]),
            "orc_exclusive_scan_u32": (None, [vp, vp, i64]),
            "orc_cell_indices_ref": (None, [vp, i64, i64, vp, vp]),
            "orc_cell_offsets": (None, [vp, i64, i64, vp, vp]),
            "orc_particles_run": (i64, [i64, vp, vp, vp, C.c_int, f32, f32, f32, f32, f32, u32, C.c_int, C.c_int]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _orc = L
    return _orc


def ref_available() -> bool:
    return os.path.exists(REF_LIB)


def ref():
    global _ref
    if _ref is None:
        L = C.CDLL(REF_LIB)
        sig = {
            "gref_set_model": (None, [C.c_int, C.c_int, C.c_int, f32, f32, vp]),
            "gref_homog_diffuse": (None, [vp, vp, C.c_int, C.c_int]),
            "gref_source_boundary": (None, [vp, C.c_int, C.c_int, C.c_int, C.c_int]),
            "gref_inhomog_diffuse": (None, [vp, vp, vp, vp, vp, vp, C.c_int, C.c_int, f32, C.c_int]),
            "gref_timestep_cells": (None, [vp, vp, vp, vp, C.c_int, C.c_int, vp]),
            "gref_det_diffuse_inplace": (None, [vp, vp, f32]),
            "gref_threefry2x32": (None, [vp, vp, vp]),
            "gref_philox4x32": (None, [vp, vp, vp]),
        }
        # model-specific kernels generated from the reference's templates (ref/gen_models.py)
        for m in ("abc", "dimer", "abcloc"):
            sig[f"gref_ssa_{m}"] = (None, [vp, C.c_int, f32, vp])
        for m in ("gs", "gsloc"):
            sig[f"gref_rk4_{m}"] = (None, [vp, f32, vp])
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _ref = L
    return _ref


def model_ptr(desc):
    """desc: a ctypes structure with the gpgmp_model_desc layout."""
    return C.cast(C.pointer(desc), C.c_void_p)


# ---- convenience wrappers -----------------------------------------------------------

def rep_solve(desc, state: np.ndarray, R: int, seed: int, max_snaps: int):
    st = np.ascontiguousarray(state, dtype=np.int32).copy()
    snaps = np.zeros((max_snaps,) + st.shape, dtype=np.int32)
    times = np.zeros(max_snaps, dtype=np.float32)
    ns = C.c_int(0)
    steps = C.c_int64(0)
    status = np.zeros(R, dtype=np.int32)
    orc().orc_rep_solve(model_ptr(desc), ptr(st), R, seed, ptr(snaps), ptr(times), max_snaps, C.byref(ns),
                        C.byref(steps), ptr(status))
    n = min(ns.value, max_snaps)
    return st, snaps[:n], times[:n], steps.value, status


def ref_solve(desc, state: np.ndarray, seed_base: int, max_snaps: int):
    st = np.ascontiguousarray(state, dtype=np.int32).copy()
    snaps = np.zeros((max_snaps,) + st.shape, dtype=np.int32)
    times = np.zeros(max_snaps, dtype=np.float32)
    ns = C.c_int(0)
    steps = C.c_int64(0)
    orc().orc_ref_solve(model_ptr(desc), ptr(st), seed_base, ptr(snaps), ptr(times), max_snaps, C.byref(ns),
                        C.byref(steps))
    n = min(ns.value, max_snaps)
    return st, snaps[:n], times[:n], steps.value


def init_poisson(W, H, S, R, seed, lam):
    out = np.zeros((R, S, H, W), dtype=np.int32)
    lam = np.ascontiguousarray(lam, dtype=np.float32)
    orc().orc_rep_init_poisson(W, H, S, R, seed, ptr(lam), ptr(out))
    return out


HAZARD_FN = C.CFUNCTYPE(C.c_float, C.c_int, C.POINTER(C.c_int32))


def set_custom_hazard(fn):
    """fn(r, counts) -> float32 hazard for the replay's SSA (None: mass action).
    Returns the ctypes callback object, which the caller keeps alive while in use."""
    if fn is None:
        orc().orc_set_custom_hazard(None)
        return None
    cb = HAZARD_FN(lambda r, x: float(fn(r, x)))
    orc().orc_set_custom_hazard(C.cast(cb, C.c_void_p))
    return cb
