"""Loads micm_b200/libmicmb.so and declares the C ABI of include/micmb.h.

The library must have been built (``python -c "import __graft_entry__ as g; g.build()"``
or ``make -C micm_b200/csrc``); there is no fallback implementation.
"""
from __future__ import annotations

import ctypes as C
import os

from ._abi import BackwardEulerParams, FusedConfig, MechanismDesc, MechanismInfo, RosenbrockParams, SolverStats

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmicmb.so")

_lib = None

i32p = C.POINTER(C.c_int32)
f64p = C.POINTER(C.c_double)
vp = C.c_void_p


class MicmbError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"[{code}] {message}")
        self.code = code


# int allgather(const double* send, double* recv, int32_t world, void* stream, void* user)
ALLGATHER_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with make -C micm_b200/csrc")
        L = C.CDLL(LIB_PATH)
        L.micmb_last_error.restype = C.c_char_p
        sig = {
            "micmb_mechanism_create": [C.POINTER(MechanismDesc), C.POINTER(vp)],
            "micmb_mechanism_get_info": [vp, C.POINTER(MechanismInfo)],
            "micmb_mechanism_species_columns": [vp, i32p],
            "micmb_mechanism_reaction_columns": [vp, i32p],
            "micmb_mechanism_custom_param_columns": [vp, i32p],
            "micmb_mechanism_jacobian_pattern": [vp, i32p, i32p],
            "micmb_mechanism_jacobian_pattern_unfilled": [vp, i32p, i32p],
            "micmb_rosenbrock_params_default": [C.c_int32, C.POINTER(RosenbrockParams)],
            "micmb_mechanism_stream_stats": [vp, C.POINTER(C.c_int64)],
            "micmb_solver_create": [vp, C.POINTER(RosenbrockParams), C.POINTER(vp)],
            "micmb_solver_set_params": [vp, C.POINTER(RosenbrockParams)],
            "micmb_solver_set_rate_scale": [vp, f64p],
            "micmb_solver_set_fused_config": [vp, C.POINTER(FusedConfig)],
            "micmb_solver_get_fused_config": [vp, C.POINTER(FusedConfig)],
            "micmb_state_create": [vp, C.c_int64, C.c_int32, C.POINTER(vp)],
            "micmb_state_set_stream": [vp, vp],
            "micmb_state_synchronize": [vp],
            "micmb_state_upload": [vp, C.c_int32, f64p],
            "micmb_state_download": [vp, C.c_int32, f64p],
            "micmb_state_device_buffer": [vp, C.c_int32, C.POINTER(f64p), C.POINTER(C.c_int64)],
            "micmb_state_set_relative_tolerance": [vp, C.c_double],
            "micmb_update_state_parameters": [vp, vp],
            "micmb_solve": [vp, vp, C.c_double, C.c_int32, C.c_int32, C.POINTER(SolverStats), i32p, i32p],
            "micmb_autotune": [vp, vp, C.c_double, C.c_char_p, C.POINTER(FusedConfig)],
            "micmb_solve_graph": [vp, vp, C.c_double, C.c_int32],
            "micmb_solve_adjoint": [vp, vp, C.c_double, f64p, f64p, f64p, C.c_int32, C.POINTER(SolverStats)],
            "micmb_set_adjoint_memory_limit": [vp, C.c_int64],
            "micmb_add_forcing_terms": [vp, vp],
            "micmb_subtract_jacobian_terms": [vp, vp],
            "micmb_alpha_minus_jacobian": [vp, vp, C.c_double],
            "micmb_lu_decompose": [vp, vp],
            "micmb_linear_solve": [vp, vp],
            "micmb_normalized_error": [vp, vp, f64p, f64p],
            "micmb_normalized_error_noalloc": [vp, vp, f64p],
            "micmb_math_eval": [C.c_int32, vp, vp, vp, C.c_int64, C.c_int32],
            "micmb_state_set_global_exchange": [vp, ALLGATHER_FN, vp, C.c_int32, C.c_int64],
            "micmb_backward_euler_params_default": [C.POINTER(BackwardEulerParams)],
            "micmb_solve_backward_euler": [vp, vp, C.c_double, C.POINTER(BackwardEulerParams), C.c_int32,
                                           C.POINTER(SolverStats), i32p, i32p],
        }
        for name, args in sig.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = C.c_int
        L.micmb_mechanism_destroy.argtypes = [vp]
        L.micmb_mechanism_destroy.restype = None
        L.micmb_solver_destroy.argtypes = [vp]
        L.micmb_solver_destroy.restype = None
        L.micmb_state_destroy.argtypes = [vp]
        L.micmb_state_destroy.restype = None
        L.micmb_mechanism_hash.argtypes = [vp]
        L.micmb_mechanism_hash.restype = C.c_uint64
        _lib = L
    return _lib


def check(rc: int):
    if rc != 0:
        raise MicmbError(rc, lib().micmb_last_error().decode())
