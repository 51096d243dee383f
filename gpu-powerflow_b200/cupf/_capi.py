"""ctypes bindings of include/cupf_b200.h (libcupf_b200.so, built in-tree).

The library is the product path: importing this module fails loudly when it
has not been built; there is no fallback implementation.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libcupf_b200.so"


class ClsConfig(C.Structure):
    _fields_ = [("precision", C.c_int32), ("matching", C.c_int32), ("pivot_strategy", C.c_int32),
                ("serial_nd", C.c_int32), ("max_panel_width", C.c_int32), ("shift_retry_epsilon", C.c_double),
                ("autotune", C.c_int32), ("parallel_nd_depth", C.c_int32), ("parallel_nd_base_small", C.c_int32),
                ("parallel_nd_base_large", C.c_int32), ("wide_min_front", C.c_int32), ("tc_min_front", C.c_int32),
                ("batch1_schedule", C.c_int32)]


class PfOptions(C.Structure):
    _fields_ = [("backend", C.c_int32), ("compute", C.c_int32), ("cuda_linear_solver", C.c_int32),
                ("cuda_jacobian", C.c_int32), ("custom", ClsConfig), ("use_cuda_graph", C.c_int32)]


class PfNRConfig(C.Structure):
    _fields_ = [("tolerance", C.c_double), ("max_iter", C.c_int32)]


class PfSolveOptions(C.Structure):
    _fields_ = [("prepare_adjoint_cache", C.c_int32), ("adjoint_cache_mode", C.c_int32),
                ("allow_explicit_transpose_fallback", C.c_int32)]


class PfAdjointOptions(C.Structure):
    _fields_ = [(n, C.c_int32) for n in (
        "reuse_forward_factorization", "allow_refactorize", "require_cached_factorization",
        "allow_refactorize_for_backward", "allow_inexact_last_newton_factorization", "use_transpose_solve",
        "allow_explicit_transpose_fallback", "compute_load_gradients", "check_residual")]


class PfAdjointResult(C.Structure):
    _fields_ = [("n_bus", C.c_int32), ("batch_size", C.c_int32), ("dim_f", C.c_int32),
                ("success", C.c_int32), ("used_adjoint_cache", C.c_int32),
                ("reused_final_state_factorization", C.c_int32), ("refactorized_for_backward", C.c_int32),
                ("iterations", C.c_int32), ("jt_residual_norm", C.c_double),
                ("max_final_mismatch", C.c_double), ("all_converged", C.c_int32)]


class PfInfo(C.Structure):
    _fields_ = [("n_bus", C.c_int32), ("n_pv", C.c_int32), ("n_pq", C.c_int32), ("dim_f", C.c_int32),
                ("nnz_ybus", C.c_int32), ("nnz_jacobian", C.c_int32), ("num_panels", C.c_int32),
                ("num_levels", C.c_int32), ("max_front", C.c_int32), ("max_panel", C.c_int32),
                ("factor_elements", C.c_int64), ("last_kernel_launches", C.c_int64)]


# exported symbols, in the order include/cupf_b200.h declares them
EXPORTS = [
    "cls_create", "cls_destroy", "cls_set_data", "cls_analyze", "cls_analyze_host", "cls_setup", "cls_set_stream", "cls_factorize",
    "cls_factorize_static_scratch",
    "cls_solve", "cls_solve_transpose", "cls_singular_flags", "cls_status_string", "cls_last_error",
    "cls_plan_array", "cls_dump_fronts_csv",
    "pf_create", "pf_destroy", "pf_last_error", "pf_initialize", "pf_analyze_host", "pf_solve_batch", "pf_solve_batch_device",
    "pf_solve_batch_ybus", "pf_solve_batch_ybus_device",
    "pf_solve_batch_warm_device", "pf_solve_forward_device", "pf_solve_backward_device", "pf_solve_adjoint",
    "pf_info", "pf_plan_array", "pf_dump_fronts_csv",
    "pf_evaluate", "pf_set_profiling", "pf_stage_times", "pf_plan_array64", "pf_singular_flags",
    "pf_case_load", "pf_case_last_error", "pf_case_dims", "pf_case_name", "pf_case_copy", "pf_case_destroy",
]
# exported symbols of include/cupf_mlp.h (warm-start network kernels)
MLP_EXPORTS = [
    "mlp_last_error", "mlp_gemm_bf16", "mlp_error_flag", "mlp_set_wait_test", "mlp_transpose_bf16", "mlp_standardize",
    "mlp_mse_grad",
    "mlp_col_sum_bf16", "mlp_adam", "mlp_load_features", "mlp_gemm_bf16_split",
    "mlp_gram_f64", "mlp_cholesky_solve_f64", "mlp_refit_last_error",
]

_vp = C.c_void_p
_i32 = C.c_int32
_i64 = C.c_int64
_p = C.POINTER


def _declare(lib: C.CDLL) -> None:
    s = {
        "cls_create": ([_p(ClsConfig), _p(_vp)], _i32),
        "cls_destroy": ([_vp], _i32),
        "cls_set_data": ([_vp, _i32, _i32, _vp, _vp, _i32], _i32),
        "cls_analyze": ([_vp], _i32),
        "cls_analyze_host": ([_vp], _i32),
        "cls_setup": ([_vp, _i32], _i32),
        "cls_set_stream": ([_vp, _vp], _i32),
        "cls_factorize": ([_vp, _vp, _i32], _i32),
        "cls_factorize_static_scratch": ([_vp, _vp, _i32], _i32),
        "cls_solve": ([_vp, _vp, _i32, _vp, _i32], _i32),
        "cls_solve_transpose": ([_vp, _vp, _i32, _vp, _i32], _i32),
        "cls_singular_flags": ([_vp, _vp, _i32], _i32),
        "cls_status_string": ([_i32], C.c_char_p),
        "cls_last_error": ([_vp], C.c_char_p),
        "cls_plan_array": ([_vp, C.c_char_p, _vp, _i64, _p(_i64)], _i32),
        "cls_dump_fronts_csv": ([_vp, C.c_char_p], _i32),
        "pf_create": ([_p(PfOptions), _p(_vp)], _i32),
        "pf_destroy": ([_vp], _i32),
        "pf_last_error": ([_vp], C.c_char_p),
        "pf_initialize": ([_vp, _vp, _vp, _vp, _i32, _i32, _i32, _vp, _i32, _vp, _i32], _i32),
        "pf_analyze_host": ([_vp, _vp, _vp, _i32, _i32, _vp, _i32, _vp, _i32], _i32),
        "pf_solve_batch": ([_vp, _vp, _vp, _vp, _i32, _i32, _i32, _vp, _i64, _vp, _i64, _i32, _vp, _i32, _vp, _i32,
                            _p(PfNRConfig), _p(PfSolveOptions), _vp, _vp, _vp, _vp], _i32),
        "pf_solve_batch_device": ([_vp, _vp, _i64, _vp, _i64, _i32, _p(PfNRConfig), _p(PfSolveOptions), _vp, _vp,
                                   _vp, _p(PfAdjointResult)], _i32),
        "pf_solve_batch_ybus": ([_vp, _vp, _i64, _vp, _i64, _vp, _i64, _i32, _p(PfNRConfig), _p(PfSolveOptions), _vp,
                                 _vp, _vp, _vp], _i32),
        "pf_solve_batch_ybus_device": ([_vp, _vp, _i64, _vp, _i64, _vp, _i64, _i32, _p(PfNRConfig),
                                        _p(PfSolveOptions), _vp, _vp, _vp, _p(PfAdjointResult)], _i32),
        "pf_solve_batch_warm_device": ([_vp, _vp, _i64, _vp, _i64, _vp, _i64, _vp, _vp, _i32, _p(PfNRConfig),
                                        _p(PfSolveOptions), _vp, _vp, _vp, _p(PfAdjointResult)], _i32),
        "pf_solve_forward_device": ([_vp, _vp, _vp, _vp, _vp, _vp, _vp, _i32, _vp, _vp, _i32, _i32, C.c_char_p,
                                     _p(PfNRConfig), _p(PfSolveOptions), _vp, _p(PfAdjointResult)], _i32),
        "pf_solve_backward_device": ([_vp, _vp, _vp, _vp, _vp, _i32, _i32, C.c_char_p, _p(PfAdjointOptions), _vp,
                                      _p(PfAdjointResult)], _i32),
        "pf_solve_adjoint": ([_vp, _vp, _i64, _vp, _i64, _i32, _vp, _i32, _vp, _i32, _p(PfAdjointOptions), _vp, _vp,
                              _vp, _p(PfAdjointResult)], _i32),
        "pf_info": ([_vp, _p(PfInfo)], _i32),
        "pf_plan_array": ([_vp, C.c_char_p, _vp, _i64, _p(_i64)], _i32),
        "pf_dump_fronts_csv": ([_vp, C.c_char_p], _i32),
        "pf_evaluate": ([_vp, _vp, _vp, _i32, _vp, _vp], _i32),
        "pf_set_profiling": ([_vp, _i32], _i32),
        "pf_plan_array64": ([_vp, C.c_char_p, _vp, _i64, _p(_i64)], _i32),
        "pf_stage_times": ([_vp, _vp, _vp], _i32),
        "pf_singular_flags": ([_vp, _vp, _i32], _i32),
        "pf_case_load": ([C.c_char_p, _p(_vp)], _i32),
        "pf_case_last_error": ([], C.c_char_p),
        "pf_case_dims": ([_vp, _p(_i32), _p(_i32), _p(_i32), _p(_i32), _p(_i32), _p(_i32)], _i32),
        "pf_case_name": ([_vp], C.c_char_p),
        "pf_case_copy": ([_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp], _i32),
        "pf_case_destroy": ([_vp], None),
        "mlp_last_error": ([], C.c_char_p),
        "mlp_gemm_bf16": ([_vp, _i64, _vp, _i64, _i32, _i32, _i32, _i32, _vp, _i64, _vp, _vp, _i64, _vp], _i32),
        "mlp_gemm_bf16_split": ([_vp, _i64, _vp, _i64, _i32, _i32, _i32, _i32, _vp, _i64, _vp, _vp], _i32),
        "mlp_error_flag": ([_p(_i32), _i32], _i32),
        "mlp_set_wait_test": ([C.c_longlong, _i32], _i32),
        "mlp_gram_f64": ([_vp, _i64, _i32, _vp, _i64, _i32, _i32, _i32, _i32, _vp, _i64, _vp, _i64, _vp], _i32),
        "mlp_cholesky_solve_f64": ([_vp, _i64, _i32, _vp, _i64, _i32, C.c_double, _vp, _vp], _i32),
        "mlp_refit_last_error": ([], C.c_char_p),
        "mlp_transpose_bf16": ([_vp, _i64, _vp, _i32, _i32, _vp], _i32),
        "mlp_standardize": ([_vp, _vp, _vp, _vp, _i64, _i32, _i32, _i32, _vp], _i32),
        "mlp_load_features": ([_vp, _i64, _vp, _vp, _i32, _i32, _vp, _vp, _vp, _i64, _i32, _i32, _i32, _vp], _i32),
        "mlp_mse_grad": ([_vp, _i32, _vp, _i32, _i32, _vp, _vp, _vp], _i32),
        "mlp_col_sum_bf16": ([_vp, _i32, _i32, _vp, _vp], _i32),
        "mlp_adam": ([_vp, _vp, _vp, _vp, _vp, _i64, C.c_float, C.c_float, C.c_float, C.c_float, _i32, C.c_float,
                      _vp], _i32),
    }
    for name, (args, res) in s.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res


_LIB: C.CDLL | None = None


def load() -> C.CDLL:
    """Load the engine library (raises if it was not built)."""
    global _LIB
    if _LIB is None:
        if not LIB_PATH.exists():
            raise ImportError(
                f"{LIB_PATH} is missing: build the CUDA engine first "
                "(python gpu-powerflow_b200/build.py or __graft_entry__.build())")
        mode = getattr(os, "RTLD_GLOBAL", 0)
        lib = C.CDLL(str(LIB_PATH), mode=mode)
        _declare(lib)
        _LIB = lib
    return _LIB
