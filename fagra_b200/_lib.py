"""ctypes binding of libfagra_b200.so (declared in include/fagra_b200.h).

The shared library is the product: there is no CPU fallback. Importing this
module without the built library raises immediately.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB_PATH = Path(os.environ.get("FAGRA_B200_LIB", HERE / "libfagra_b200.so"))

size_t = C.c_size_t
ptrdiff_t = C.c_ssize_t
dptr = C.POINTER(C.c_double)


class SchurOptions(C.Structure):
    _fields_ = [
        ("max_iterations", size_t),
        ("relative_tolerance", C.c_double),
        ("collect_timings", C.c_int),
        ("precision", C.c_int),
        ("preconditioner", C.c_int),
        ("device", C.c_int),
        ("residual_replacement", C.c_double),
        ("operator_variant", C.c_int),
        ("coarse_correction", C.c_int),
        ("learned_policy", C.c_int),
    ]


class SchurDiagnosticsC(C.Structure):
    _fields_ = [
        ("termination", C.c_int),
        ("iterations", size_t),
        ("damping", C.c_double),
        ("estimated_relative_residual", C.c_double),
        ("reduced_relative_residual", C.c_double),
        ("scaled_relative_residual", C.c_double),
        ("original_relative_residual", C.c_double),
        ("has_estimated", C.c_int),
        ("has_reduced", C.c_int),
        ("has_scaled", C.c_int),
        ("has_original", C.c_int),
        ("refinements", size_t),
        ("preconditioner_used", C.c_int),
        ("learned_fallback", C.c_int),
        ("learned_iterations", size_t),
        ("block_jacobi_iterations", size_t),
        ("learned_seconds", C.c_double),
        ("block_jacobi_seconds", C.c_double),
        ("coarse_vectors", size_t),
    ]


class SchurTimingsC(C.Structure):
    _fields_ = [(n, C.c_double) for n in
                ("preparation", "factorization", "linear_solve", "products", "preconditioner", "verification")]


class LsmrOptions(C.Structure):
    _fields_ = [
        ("max_iterations", size_t),
        ("relative_tolerance", C.c_double),
        ("diagonal_preconditioning", C.c_int),
        ("block_preconditioning", C.c_int),
        ("collect_timings", C.c_int),
        ("precision", C.c_int),
        ("device", C.c_int),
    ]


class LsmrDiagnosticsC(C.Structure):
    _fields_ = [
        ("termination", C.c_int),
        ("iterations", size_t),
        ("finite_step", C.c_int),
        ("estimated_absolute_residual", C.c_double),
        ("estimated_relative_residual", C.c_double),
        ("original_absolute_residual", C.c_double),
        ("original_relative_residual", C.c_double),
        ("scaled_absolute_residual", C.c_double),
        ("scaled_relative_residual", C.c_double),
        ("min_scale", C.c_double),
        ("max_scale", C.c_double),
        ("damping", C.c_double),
        ("block_fallbacks", size_t),
        ("has_estimated", C.c_int),
        ("has_original", C.c_int),
        ("has_scaled", C.c_int),
        ("has_scales", C.c_int),
        ("has_damping", C.c_int),
    ]


class LsmrTimingsC(C.Structure):
    _fields_ = [(n, C.c_double) for n in
                ("preparation", "factorization", "linear_solve", "forward", "transpose", "preconditioner",
                 "residual_checks")]


class WindowReportC(C.Structure):
    _fields_ = [
        ("status", C.c_int), ("termination", C.c_int),
        ("iterations", size_t), ("linearizations", size_t), ("attempts", size_t), ("rejected_steps", size_t),
        ("cost_evaluations", size_t), ("last_rejection", C.c_int),
        ("initial_cost", C.c_double), ("final_cost", C.c_double), ("damping", C.c_double),
        ("gradient_norm", C.c_double), ("step_norm", C.c_double),
        ("prior_status", C.c_int), ("prior_rows", size_t), ("eliminated_rank", size_t),
        ("separator_poses", size_t), ("prior_constant", C.c_double),
    ]


class OptimizeOptionsC(C.Structure):
    _fields_ = [
        ("max_iterations", size_t),
        ("gradient_tolerance", C.c_double),
        ("step_tolerance", C.c_double),
        ("cost_tolerance", C.c_double),
    ]


class LmOptionsC(C.Structure):
    _fields_ = [
        ("initial_damping", C.c_double),
        ("min_damping", C.c_double),
        ("max_damping", C.c_double),
        ("min_column_norm", C.c_double),
        ("acceptance_threshold", C.c_double),
        ("max_trials", size_t),
    ]


class ReportC(C.Structure):
    _fields_ = [
        ("iterations", size_t),
        ("initial_cost", C.c_double),
        ("final_cost", C.c_double),
        ("termination", C.c_int),
    ]


class LmStatisticsC(C.Structure):
    _fields_ = [
        ("linearizations", size_t),
        ("attempts", size_t),
        ("rejected_steps", size_t),
        ("accepted_steps", size_t),
        ("cost_evaluations", size_t),
        ("damping", C.c_double),
        ("cost", C.c_double),
        ("gradient_norm", C.c_double),
        ("step_norm", C.c_double),
        ("has_cost", C.c_int),
        ("has_gradient_norm", C.c_int),
        ("has_step_norm", C.c_int),
        ("last_rejection", C.c_int),
        ("linear_solves", size_t),
        ("linear_iterations", size_t),
        ("linear_work_available", C.c_int),
    ]


ACCEPT_CB = C.CFUNCTYPE(None, C.c_void_p, C.POINTER(LmStatisticsC))
COST_CB = C.CFUNCTYPE(C.c_int, C.c_void_p, dptr, dptr)
LIN_CB = C.CFUNCTYPE(C.c_int, C.c_void_p, dptr, C.c_void_p)


class ProblemCallbacksC(C.Structure):
    _fields_ = [("dimension", size_t), ("cost", COST_CB), ("linearize", LIN_CB)]


# name: (restype, argtypes)
SIGNATURES = {
    "fg_version": (C.c_char_p, []),
    "fg_last_error": (C.c_char_p, []),
    "fg_device_count": (C.c_int, [C.POINTER(C.c_int)]),
    "fg_device_stream": (C.c_int, [C.c_int, C.POINTER(C.c_void_p)]),
    "fg_kernel_launches": (C.c_uint64, []),
    "fg_schur_default_options": (None, [C.POINTER(SchurOptions)]),
    "fg_schur_create": (C.c_int, [size_t, size_t, size_t, C.POINTER(SchurOptions), C.POINTER(C.c_void_p)]),
    "fg_backend_destroy": (None, [C.c_void_p]),
    "fg_schur_set_options": (C.c_int, [C.c_void_p, C.POINTER(SchurOptions)]),
    "fg_backend_prepare": (C.c_int, [C.c_void_p, size_t]),
    "fg_backend_clear": (C.c_int, [C.c_void_p]),
    "fg_backend_accumulate": (C.c_int, [C.c_void_p, size_t, dptr, size_t, C.POINTER(size_t), C.POINTER(size_t),
                                        C.POINTER(dptr), C.POINTER(ptrdiff_t), C.POINTER(ptrdiff_t)]),
    "fg_backend_gradient_norm": (C.c_int, [C.c_void_p, dptr]),
    "fg_backend_solve": (C.c_int, [C.c_void_p, C.POINTER(dptr), C.POINTER(size_t)]),
    "fg_backend_prepare_damping": (C.c_int, [C.c_void_p, C.c_double]),
    "fg_backend_solve_damped": (C.c_int, [C.c_void_p, C.c_double, C.POINTER(dptr), C.POINTER(size_t), dptr]),
    "fg_backend_solve_damped_device": (C.c_int, [C.c_void_p, C.c_double, C.POINTER(dptr), dptr]),
    "fg_backend_linear_solve_work": (C.c_int, [C.c_void_p, C.POINTER(size_t), C.POINTER(size_t),
                                               C.POINTER(C.c_int)]),
    "fg_schur_get_diagnostics": (C.c_int, [C.c_void_p, C.POINTER(SchurDiagnosticsC)]),
    "fg_schur_get_timings": (C.c_int, [C.c_void_p, C.POINTER(SchurTimingsC)]),
    "fg_schur_structure_sizes": (C.c_int, [C.c_void_p] + [C.POINTER(size_t)] * 6),
    "fg_schur_export_structure": (C.c_int, [C.c_void_p] + [C.POINTER(C.c_uint64)] * 4),
    "fg_schur_export_model": (C.c_int, [C.c_void_p] + [dptr] * 6),
    "fg_schur_reduced_apply": (C.c_int, [C.c_void_p, C.c_double, dptr, dptr]),
    "fg_bal_create": (C.c_int, [size_t, size_t, size_t, dptr, dptr, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                                dptr, C.c_int, C.POINTER(C.c_void_p)]),
    "fg_bal_create_device": (C.c_int, [size_t, size_t, size_t, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                       C.c_void_p, C.c_int, C.POINTER(C.c_void_p)]),
    "fg_bal_destroy": (None, [C.c_void_p]),
    "fg_bal_set_parameters": (C.c_int, [C.c_void_p, dptr, dptr]),
    "fg_bal_get_parameters": (C.c_int, [C.c_void_p, dptr, dptr]),
    "fg_bal_cost": (C.c_int, [C.c_void_p, dptr]),
    "fg_bal_linearize": (C.c_int, [C.c_void_p, C.c_void_p]),
    "fg_bal_cost_noalloc": (C.c_int, [size_t, size_t, size_t, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                      C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]),
    "fg_optimize_default_options": (None, [C.POINTER(OptimizeOptionsC)]),
    "fg_lm_default_options": (None, [C.POINTER(LmOptionsC)]),
    "fg_lm_solve_bal": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(OptimizeOptionsC), C.POINTER(LmOptionsC),
                                  C.POINTER(ReportC), C.POINTER(LmStatisticsC), ACCEPT_CB, C.c_void_p]),
    "fg_lm_solve_bal_to_cost": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(OptimizeOptionsC), C.POINTER(LmOptionsC),
                                          C.c_double, C.POINTER(ReportC), C.POINTER(LmStatisticsC)]),
    "fg_bal_restore_initial": (C.c_int, [C.c_void_p]),
    "fg_schur_time_operator": (C.c_int, [C.c_void_p, C.c_double, size_t, dptr, dptr]),
    "fg_schur_time_operator_kernel": (C.c_int, [C.c_void_p, C.c_double, size_t, dptr, dptr]),
    "fg_schur_operator_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), dptr]),
    "fg_schur_set_poll_limit": (C.c_int, [C.c_void_p, C.c_uint]),
    "fg_schur_accumulate_pairs_device": (C.c_int, [C.c_void_p, size_t, size_t, C.c_void_p, C.c_void_p, C.c_void_p,
                                                   C.c_void_p, C.c_void_p]),
    "fg_gn_solve_bal": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(OptimizeOptionsC), C.POINTER(ReportC)]),
    "fg_lm_optimize": (C.c_int, [C.c_void_p, C.POINTER(ProblemCallbacksC), C.c_void_p, dptr,
                                 C.POINTER(OptimizeOptionsC), C.POINTER(LmOptionsC), C.POINTER(ReportC),
                                 C.POINTER(LmStatisticsC)]),
    "fg_gn_optimize": (C.c_int, [C.c_void_p, C.POINTER(ProblemCallbacksC), C.c_void_p, dptr,
                                 C.POINTER(OptimizeOptionsC), C.POINTER(ReportC)]),
    "fg_windows_create": (C.c_int, [size_t, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), C.POINTER(C.c_uint32),
                                    size_t, C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    "fg_windows_destroy": (None, [C.c_void_p]),
    "fg_windows_prior_layout": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64),
                                          C.POINTER(C.c_uint32)]),
    "fg_windows_set_priors": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), dptr, dptr,
                                        dptr]),
    "fg_windows_upload": (C.c_int, [C.c_void_p, dptr, dptr, dptr]),
    "fg_windows_run": (C.c_int, [C.c_void_p, C.POINTER(OptimizeOptionsC), C.POINTER(LmOptionsC)]),
    "fg_windows_download": (C.c_int, [C.c_void_p, dptr, C.POINTER(WindowReportC), dptr, dptr]),
    "fg_windows_solve": (C.c_int, [C.c_void_p, dptr, dptr, dptr, C.POINTER(OptimizeOptionsC), C.POINTER(LmOptionsC),
                                   C.POINTER(WindowReportC), dptr, dptr]),
    "fg_windows_tuning": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int), dptr]),
    "fg_windows_stream": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "fg_dense_normal_create": (C.c_int, [C.c_int, C.POINTER(C.c_void_p)]),
    "fg_dense_schur_create": (C.c_int, [size_t, C.POINTER(size_t), size_t, C.c_int, C.POINTER(C.c_void_p)]),
    "fg_dense_qr_create": (C.c_int, [C.c_double, C.c_int, C.POINTER(C.c_void_p)]),
    "fg_dense_qr_set_tolerance": (C.c_int, [C.c_void_p, C.c_double]),
    "fg_backend_covariance": (C.c_int, [C.c_void_p, C.POINTER(size_t), size_t, C.c_double, dptr]),
    "fg_lsmr_default_options": (None, [C.POINTER(LsmrOptions)]),
    "fg_lsmr_create": (C.c_int, [C.POINTER(LsmrOptions), C.POINTER(C.c_void_p)]),
    "fg_lsmr_set_options": (C.c_int, [C.c_void_p, C.POINTER(LsmrOptions)]),
    "fg_lsmr_get_diagnostics": (C.c_int, [C.c_void_p, C.POINTER(LsmrDiagnosticsC)]),
    "fg_lsmr_get_timings": (C.c_int, [C.c_void_p, C.POINTER(LsmrTimingsC)]),
    "fg_lsmr_damped_products": (C.c_int, [C.c_void_p, C.c_double, C.c_int, dptr, dptr, dptr, dptr]),
    "fg_lsmr_time_iteration": (C.c_int, [C.c_void_p, C.c_double, size_t, dptr, dptr]),
    "fg_gnn_create": (C.c_int, [C.c_uint64, C.c_int, C.POINTER(C.c_void_p)]),
    "fg_gnn_destroy": (None, [C.c_void_p]),
    "fg_gnn_parameter_count": (C.c_int, [C.c_void_p, C.POINTER(size_t)]),
    "fg_gnn_get_parameters": (C.c_int, [C.c_void_p, C.POINTER(C.c_float)]),
    "fg_gnn_set_parameters": (C.c_int, [C.c_void_p, C.POINTER(C.c_float)]),
    "fg_schur_capture_system": (C.c_int, [C.c_void_p, C.c_void_p, C.c_double, size_t, C.c_uint64, C.c_int,
                                          C.POINTER(size_t)]),
    "fg_gnn_import_system": (C.c_int, [C.c_void_p, size_t, size_t, size_t, C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float),
                                       C.POINTER(C.c_uint8), C.POINTER(size_t)]),
    "fg_gnn_system_count": (C.c_int, [C.c_void_p, C.POINTER(size_t)]),
    "fg_gnn_system_size": (C.c_int, [C.c_void_p, size_t, C.POINTER(size_t), C.POINTER(size_t), C.POINTER(size_t)]),
    "fg_gnn_export_system": (C.c_int, [C.c_void_p, size_t, C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_uint8), dptr]),
    "fg_gnn_clear_systems": (C.c_int, [C.c_void_p]),
    "fg_gnn_evaluate": (C.c_int, [C.c_void_p, size_t, dptr, C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "fg_gnn_train": (C.c_int, [C.c_void_p, size_t, C.c_double, dptr]),
    "fg_schur_attach_learned": (C.c_int, [C.c_void_p, C.c_void_p]),
}


def _load() -> C.CDLL:
    if not LIB_PATH.exists():
        raise ImportError(
            f"fagra_b200: CUDA library {LIB_PATH} is missing; build it with `python -m fagra_b200.build` "
            "(there is no CPU fallback)")
    lib = C.CDLL(str(LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def last_error() -> str:
    return (lib.fg_last_error() or b"").decode()


def device_count() -> int:
    n = C.c_int(0)
    lib.fg_device_count(C.byref(n))
    return n.value


def kernel_launches() -> int:
    return int(lib.fg_kernel_launches())


def device_stream(device: int = 0) -> int:
    s = C.c_void_p()
    _check(lib.fg_device_stream(device, C.byref(s)))
    return s.value or 0


from .errors import raise_for_status as _check  # noqa: E402
