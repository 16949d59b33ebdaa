"""Loader of the in-tree C-ABI library ``libtensors_b200.so``.

The library is required: there is no CPU fallback for the numeric path.  If
the shared object is missing, importing :func:`lib` raises with the build
command to run.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtensors_b200.so")

# every entry point declared in include/tensors_b200.h
_vp = ctypes.c_void_p
_i32 = ctypes.c_int32
_i64 = ctypes.c_int64
_d = ctypes.c_double
_pi32 = ctypes.POINTER(ctypes.c_int32)
_pi64 = ctypes.POINTER(ctypes.c_int64)
_pd = ctypes.POINTER(ctypes.c_double)

SIGNATURES = {
    "tb_last_error": (ctypes.c_char_p, []),
    "tb_trace_record": (ctypes.c_int, [_i32]),
    "tb_trace_names": (ctypes.c_int64, [ctypes.c_char_p, ctypes.c_int64]),
    "tb_trace_times": (ctypes.c_int64, [ctypes.POINTER(ctypes.c_double), ctypes.c_int64]),
    "tb_set_device": (ctypes.c_int, [ctypes.c_int]),
    "tb_chol_create": (ctypes.c_int, [ctypes.POINTER(_vp), _i32, _vp, _vp, _vp, _i32]),
    "tb_chol_destroy": (ctypes.c_int, [_vp]),
    "tb_chol_set_supernode_strategy": (ctypes.c_int, [_vp, _i32]),
    "tb_chol_set_amalgamation_threshold": (ctypes.c_int, [_vp, _i32]),
    "tb_chol_set_factorization_method": (ctypes.c_int, [_vp, _i32]),
    "tb_chol_symbolic": (ctypes.c_int, [_vp]),
    "tb_chol_numeric": (ctypes.c_int, [_vp, _vp, _d]),
    "tb_chol_numeric_device": (ctypes.c_int, [_vp, _vp, _d]),
    "tb_chol_solve": (ctypes.c_int, [_vp, _d, _vp, _i32, _d, _vp, _i32, _i32]),
    "tb_chol_solve_device": (ctypes.c_int, [_vp, _d, _vp, _i32, _d, _vp, _i32, _i32]),
    "tb_chol_solve_device_noalloc": (ctypes.c_int, [_vp, _d, _vp, _i32, _d, _vp, _i32, _i32]),
    "tb_chol_numeric_ex": (ctypes.c_int, [_vp, _vp, _i32, _d]),
    "tb_chol_set_plan_options": (ctypes.c_int, [_vp, _i32, _i32, _i32]),
    "tb_chol_gmres": (ctypes.c_int, [_vp, _vp, _d, _d, _vp, _i32, _d, _vp, _i32, _i32, _d, _i32, _i32, _i32, _pi32, _pi32, _vp]),
    "tb_chol_gmres_device": (ctypes.c_int, [_vp, _vp, _d, _d, _vp, _i32, _d, _vp, _i32, _i32, _d, _i32, _i32, _i32, _pi32, _pi32, _vp]),
    "tb_chol_gmres_ir_iterations": (ctypes.c_int, [_vp, _pi32]),
    "tb_chol_plan_options": (ctypes.c_int, [_vp, _pi32, _pi32, _pi32]),
    "tb_chol_autotune_plan": (ctypes.c_int, [_vp, _pi32, _pd, _i32]),
    "tb_chol_numeric_device_ex": (ctypes.c_int, [_vp, _vp, _i32, _d]),
    "tb_chol_solve_ex": (ctypes.c_int, [_vp, _d, _vp, _i32, _i32, _d, _vp, _i32, _i32, _i32]),
    "tb_chol_solve_device_ex": (ctypes.c_int, [_vp, _d, _vp, _i32, _i32, _d, _vp, _i32, _i32, _i32]),
    "tb_factor_create": (ctypes.c_int, [ctypes.POINTER(_vp)]),
    "tb_factor_destroy": (ctypes.c_int, [_vp]),
    "tb_factor_state": (ctypes.c_int, [_vp, _pi32, _pi32, _pi64, _pi32]),
    "tb_chol_swap_factor": (ctypes.c_int, [_vp, _vp]),
    "tb_chol_upper_solve": (ctypes.c_int, [_vp, _d, _vp, _i32, _d, _vp, _i32, _i32]),
    "tb_chol_lower_solve": (ctypes.c_int, [_vp, _d, _vp, _i32, _d, _vp, _i32, _i32]),
    "tb_chol_residual_device": (ctypes.c_int, [_vp, _vp, _vp, _vp, _i32]),
    "tb_chol_sn_count": (ctypes.c_int, [_vp, _pi32]),
    "tb_chol_row_count": (ctypes.c_int, [_vp, _pi32]),
    "tb_chol_nonzero_count": (ctypes.c_int, [_vp, _pi64]),
    "tb_chol_array_size": (ctypes.c_int, [_vp, _i32, _pi64]),
    "tb_chol_array_copy": (ctypes.c_int, [_vp, _i32, _vp]),
    "tb_chol_factorized": (ctypes.c_int, [_vp, _pi32, _pi32]),
    "tb_chol_failed_supernode": (ctypes.c_int, [_vp, _pi32]),
    "tb_chol_factor_sizes": (ctypes.c_int, [_vp, _pi64, _pi64]),
    "tb_chol_factor_values": (ctypes.c_int, [_vp, _vp, _vp]),
    "tb_chol_log_det": (ctypes.c_int, [_vp, _pd]),
    "tb_chol_u_nonzero_count": (ctypes.c_int, [_vp, _pi64]),
    "tb_chol_get_u": (ctypes.c_int, [_vp, _vp, _vp, _vp]),
    "tb_chol_factor_diagonal": (ctypes.c_int, [_vp, _vp]),
    "tb_chol_flop_count": (ctypes.c_int, [_vp, _pd, _pd]),
    "tb_chol_device_bytes": (ctypes.c_int, [_vp, _pi64]),
    "tb_chol_plan_stats": (ctypes.c_int, [_vp, _vp, _i32]),
    "tb_chol_check_plan": (ctypes.c_int, [_vp]),
    "tb_chol_set_stream": (ctypes.c_int, [_vp, _vp]),
    "tb_chol_set_graph": (ctypes.c_int, [_vp, _i32]),
    "tb_chol_solve_profile": (ctypes.c_int, [_vp, _vp, _vp, _i32]),
    "tb_chol_launch_counts": (ctypes.c_int, [_vp, _pi64, _pi64]),
    "tb_chol_cg": (ctypes.c_int, [_vp, _vp, _d, _d, _vp, _i32, _d, _vp, _i32, _i32, _d, _i32, _i32, _pi32, _vp]),
    "tb_chol_cg_device": (ctypes.c_int, [_vp, _vp, _d, _d, _vp, _i32, _d, _vp, _i32, _i32, _d, _i32, _i32, _pi32, _vp]),
    "tb_chol_set_schedule": (ctypes.c_int, [_vp, _i32]),
    "tb_chol_set_solve_schedule": (ctypes.c_int, [_vp, _i32]),
    "tb_chol_autotune": (ctypes.c_int, [_vp, _i32, _vp, _vp]),
    "tb_chol_set_trace": (ctypes.c_int, [_vp, _i32]),
    "tb_chol_trace": (ctypes.c_int, [_vp, _vp, ctypes.c_int64]),
    "tb_chol_solve_trace": (ctypes.c_int, [_vp, _vp, ctypes.c_int64]),
    "tb_chol_set_precision": (ctypes.c_int, [_vp, _i32]),
    "tb_chol_set_refinement": (ctypes.c_int, [_vp, _d, _i32]),
    "tb_chol_refinement_info": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_double)]),
    "tb_chol_perturbed_pivots": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_int32)]),
    "tb_chol_precision_in_use": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32)]),
    "tb_chol_set_profiling": (ctypes.c_int, [_vp, _i32]),
    "tb_chol_kernel_profile": (ctypes.c_int, [_vp, _vp, _vp, _vp]),
    "tb_chol_launch_profile": (ctypes.c_int, [_vp, _vp, _vp, _i32]),
    "tb_batch_create": (ctypes.c_int, [ctypes.POINTER(_vp), _i32, _vp, _vp, _vp, _vp, _i32]),
    "tb_batch_destroy": (ctypes.c_int, [_vp]),
    "tb_batch_handle": (ctypes.c_int, [_vp, ctypes.POINTER(_vp)]),
    "tb_batch_count": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_int32)]),
    "tb_batch_offsets": (ctypes.c_int, [_vp, _vp, _vp]),
    "tb_batch_numeric": (ctypes.c_int, [_vp, _vp, _d]),
    "tb_batch_numeric_device": (ctypes.c_int, [_vp, _vp, _d]),
    "tb_batch_failed_system": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_int32)]),
    "tb_batch_solve": (ctypes.c_int, [_vp, _vp, _vp, _i32]),
    "tb_batch_solve_device": (ctypes.c_int, [_vp, _vp, _vp, _i32]),
    "tb_server_create": (ctypes.c_int, [ctypes.POINTER(_vp), ctypes.c_int, _i64, _i32, _i32]),
    "tb_server_destroy": (ctypes.c_int, [_vp]),
    "tb_server_add_matrix": (ctypes.c_int, [_vp, _i32, _vp, _vp, _vp, _i64, _pi64]),
    "tb_server_submit": (ctypes.c_int, [_vp, _i64, _vp, _d, _vp, _vp, _i32, _d, _pi64]),
    "tb_server_wait": (ctypes.c_int, [_vp, _i64, _pi32, _pd, _pd, _pi32, _pd]),
    "tb_server_stats": (ctypes.c_int, [_vp, _pi64, _pi64, _pi64, _pi64]),
    "tb_matrix_market_read": (ctypes.c_int, [ctypes.c_char_p, _i32, _pi32, _pi32, ctypes.POINTER(_pi64),
                                             ctypes.POINTER(_pi32), ctypes.POINTER(_pd)]),
    "tb_matrix_market_free": (ctypes.c_int, [_vp]),
    "tb_nested_dissection": (ctypes.c_int, [_i32, _vp, _vp, _i32, _i32, _i32, _vp]),
    "tb_matrix_market_write": (ctypes.c_int, [ctypes.c_char_p, _i32, _i32, _vp, _vp, _vp]),
}

_LIB = None


def lib() -> ctypes.CDLL:
    """The loaded library with argument/return types set (raises if absent)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing; build it with `python -m tensors_b200.build` "
                "(there is no CPU fallback for the Cholesky kernels)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _LIB = L
    return _LIB


def declared_symbols(header: str | None = None) -> list[str]:
    """Function names declared in include/tensors_b200.h."""
    import re

    header = header or os.path.join(HERE, "..", "include", "tensors_b200.h")
    text = open(header).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char \*)\s+(tb_\w+)\s*\(", text, re.M)))
