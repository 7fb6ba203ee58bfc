"""ctypes binding of libgpgmp_b200.so (the C ABI declared in include/gpgmp_c.h).

The library is built in-tree (python -m inchman_b200.build).  There is no
fallback: if the library is missing or a call fails, an exception says so.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgpgmp_b200.so")

GPGMP_OK = 0
ERRORS = {1: "invalid argument", 2: "CUDA error", 3: "out of device memory", 4: "unsupported", 5: "timeout"}

STOCHASTIC_HOMOGENEOUS = 0
STOCHASTIC_INHOMOGENEOUS = 1
DETERMINISTIC_RK4 = 2
STOCHASTIC_INHOMOGENEOUS_FPE = 3
DETERMINISTIC_AQSS = 4
DETERMINISTIC_INHOMOGENEOUS_RK4 = 5
DETERMINISTIC_INHOMOGENEOUS_AQSS = 6
DETERMINISTIC_TYPES = (DETERMINISTIC_RK4, DETERMINISTIC_AQSS, DETERMINISTIC_INHOMOGENEOUS_RK4,
                       DETERMINISTIC_INHOMOGENEOUS_AQSS)
INHOMOGENEOUS_TYPES = (STOCHASTIC_INHOMOGENEOUS, STOCHASTIC_INHOMOGENEOUS_FPE, DETERMINISTIC_INHOMOGENEOUS_RK4,
                       DETERMINISTIC_INHOMOGENEOUS_AQSS)

DRIFT_FIELD = -1
DRIFT_HOMOGENEOUS = 0
DRIFT_MULTIPLICATIVE_NOISE = 1
DRIFT_ORNSTEIN_UHLENBECK = 2
DRIFT_CODE = 3

FLAG_NONLINEAR = 1
FLAG_COMPUTE_MOMENTS = 2
FLAG_STOP_ON_ERROR = 4
FLAG_LITERAL_REDIFFUSION = 8
FLAG_AQSS_LITERAL = 16
FLAG_NO_INHOM_DET_REACTIONS = 32
CREATE_SYNC_EACH_LAUNCH = 1

SIM_EVENT_CAP = 1
SIM_OVERFLOW = 2


class Reaction(C.Structure):
    _fields_ = [
        ("rate", C.c_float),
        ("num_reactants", C.c_int32),
        ("reactant_species", C.c_int32 * 3),
        ("reactant_stoich", C.c_int32 * 3),
        ("num_products", C.c_int32),
        ("product_species", C.c_int32 * 4),
        ("product_stoich", C.c_int32 * 4),
    ]


class ModelDesc(C.Structure):
    _fields_ = [
        ("width", C.c_int32), ("height", C.c_int32), ("num_species", C.c_int32), ("num_reactions", C.c_int32),
        ("physical_length", C.c_float), ("p0", C.c_float), ("max_time", C.c_float), ("output_interval", C.c_float),
        ("max_steps", C.c_int32),
        ("boundary_mask", C.c_int32 * 4),
        ("source_mask", C.c_int32 * 4),
        ("solver_type", C.c_int32),
        ("drift_method", C.c_int32),
        ("flags", C.c_int32),
        ("drift_params", C.c_float * 8),
        ("diffusion", C.POINTER(C.c_float)),
        ("reactions", C.POINTER(Reaction)),
        ("field_dx", C.POINTER(C.c_float)),
        ("field_dy", C.POINTER(C.c_float)),
        ("field_rx", C.POINTER(C.c_float)),
        ("field_ry", C.POINTER(C.c_float)),
        ("code_defines", C.c_char_p),
        ("drift_code", C.c_char_p),
        ("custom_laws", C.POINTER(C.c_char_p)),
        ("individual", C.POINTER(C.c_uint8)),
        ("individual_capacity", C.c_int64),
        ("new_individuals_code", C.c_char_p),
        ("num_fields", C.c_int32),
        ("field_values", C.POINTER(C.c_float)),
        ("set_field_code", C.c_char_p),
        ("reaction_mask", C.POINTER(C.c_uint8)),
    ]


# int (*)(void* user, int32_t index, float time)
DUMP_CALLBACK = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int32, C.c_float)


class GpgmpError(RuntimeError):
    def __init__(self, code: int, func: str, msg: str):
        super().__init__(f"{func} failed ({ERRORS.get(code, code)}): {msg}")
        self.code = code


_lib = None
_lock = threading.Lock()

vp = C.c_void_p
i32 = C.c_int32
u32 = C.c_uint32
f32 = C.c_float
i64 = C.c_int64
P = C.POINTER

# name -> (restype, argtypes); every function in include/*.h
SIGNATURES = {
    "gpgmp_last_error": (C.c_char_p, []),
    "gpgmp_version": (C.c_int, []),
    "gpgmp_solver_create": (C.c_int, [P(ModelDesc), i32, u32, i32, P(vp)]),
    "gpgmp_solver_destroy": (C.c_int, [vp]),
    "gpgmp_solver_set_stream": (C.c_int, [vp, vp]),
    "gpgmp_set_state": (C.c_int, [vp, vp]),
    "gpgmp_get_state": (C.c_int, [vp, vp]),
    "gpgmp_init_poisson": (C.c_int, [vp, P(f32)]),
    "gpgmp_do_reactions": (C.c_int, [vp, f32, P(i32)]),
    "gpgmp_diffuse": (C.c_int, [vp, i32, f32, P(i32)]),
    "gpgmp_next_diffusion_time": (C.c_int, [vp, P(f32)]),
    "gpgmp_solve": (C.c_int, [vp, vp, P(f32), i32, P(i32), P(i64)]),
    "gpgmp_get_status": (C.c_int, [vp, P(i32)]),
    "gpgmp_synchronize": (C.c_int, [vp]),
    "gpgmp_device_state": (vp, [vp]),
    "gpgmp_timesteps": (C.c_int, [vp, P(f32), P(f32)]),
    "gpgmp_individual_count": (C.c_int, [vp, i32, P(i64)]),
    "gpgmp_update_fields": (C.c_int, [vp, f32, f32]),
    "gpgmp_get_fields": (C.c_int, [vp, P(f32)]),
    "gpgmp_set_fields": (C.c_int, [vp, P(f32)]),
    "gpgmp_solve_with_callback": (C.c_int, [vp, vp, P(f32), i32, P(i32), P(i64), vp, vp]),
    "gpgmp_get_individuals": (C.c_int, [vp, i32, vp, vp, vp, i64, P(i64)]),
    "gpgmp_set_individual_properties": (C.c_int, [vp, i32, vp, i64, i64]),
    "gpgmp_solver_launch_choices": (C.c_int, [P(i32), P(i32), P(i32), P(i32), P(i32)]),
    "gpgmp_solver_set_launch": (C.c_int, [vp, i32, i32, i32]),
    "gpgmp_solver_get_launch": (C.c_int, [vp, P(i32), P(i32), P(i32)]),
    "gpgmp_solver_autotune": (C.c_int, [vp, f32, i32, P(f32), P(f32)]),
}


def lib():
    """Loads the library once; raises if it is absent."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m inchman_b200.build`")
            L = C.CDLL(LIB_PATH)
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(L, name, None)
                if fn is None:
                    continue
                fn.restype = res
                fn.argtypes = args
            _lib = L
    return _lib


def check(code: int, func: str):
    if code != GPGMP_OK:
        msg = lib().gpgmp_last_error()
        raise GpgmpError(code, func, msg.decode() if msg else "")


def call(name: str, *args):
    code = getattr(lib(), name)(*args)
    check(code, name)
    return code
