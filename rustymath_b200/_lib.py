"""ctypes binding of librm_cuda.so (include/rm_cuda.h).

The library is required: importing the compute functions without it raises, so no call
can silently run anywhere but the B200 kernels."""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "librm_cuda.so")

RM_OK, RM_BAD_ARG, RM_NOT_REGULAR, RM_CUDA_ERROR = 0, 1, 2, 3
RM_TIMEOUT, RM_NO_CONVERGENCE, RM_NO_DEVICE, RM_OUT_OF_MEMORY = 4, 5, 6, 7
RM_NOT_POSITIVE_DEFINITE = 8
RM_METHOD_PLAIN_F64, RM_METHOD_F32_IR, RM_METHOD_GMRES_IR = 0, 1, 2
RM_INJECT_OUT_OF_MEMORY, RM_INJECT_CUDA_ERROR = 1, 2

_i32, _i64, _f64, _p = ctypes.c_int32, ctypes.c_int64, ctypes.c_double, ctypes.c_void_p


class SolveOptions(ctypes.Structure):
    _fields_ = [("method", _i32), ("max_iterations", _i32), ("gmres_restart", _i32), ("fallback", _i32),
                ("tolerance", _f64)]


class SolveReport(ctypes.Structure):
    _fields_ = [("backward_error", _f64), ("iterations", _i32), ("method_used", _i32), ("fell_back", _i32),
                ("regular", _i32)]


class BatchReport(ctypes.Structure):
    _fields_ = [("max_backward_error", _f64), ("fell_back", _i64), ("not_regular", _i64),
                ("no_convergence", _i64), ("max_iterations", _i32)]


RM_BATCH_FELL_BACK, RM_BATCH_NOT_REGULAR, RM_BATCH_NO_CONVERGENCE = 1, 2, 4


# name -> (restype, argtypes); the set of exported entry points the header declares.
SIGNATURES = {
    "rm_version": (ctypes.c_int, []),
    "rm_launch_count": (_i64, []),
    "rm_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "rm_last_error": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_size_t]),
    "rm_device_count": (ctypes.c_int, [ctypes.POINTER(ctypes.c_int)]),
    "rm_take_status": (ctypes.c_int, [_p]),
    "rm_test_inject_failure": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "rm_test_chain_timeout": (ctypes.c_int, [_i64]),
    "rm_dgemm": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _i64, _i64, _i64, _f64, _p, _i64, _p, _i64, _f64, _p,
                                _i64, _p]),
    "rm_dgemm_host": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _i64, _i64, _i64, _f64, _p, _i64, _p, _i64, _f64,
                                     _p, _i64]),
    "rm_sgemm_tc": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _i64, _i64, _i64, ctypes.c_float, _p, _i64, _p, _i64,
                                   ctypes.c_float, _p, _i64, _p]),
    "rm_dlu_factor": (ctypes.c_int, [_i64, _p, _p, _p, ctypes.POINTER(_i32), _p]),
    "rm_dlu_factor_host": (ctypes.c_int, [_i64, _p, _p, _p, ctypes.POINTER(_i32)]),
    "rm_dlu_solve": (ctypes.c_int, [_i64, _p, _p, _p, _i64, _p, ctypes.c_int, _p]),
    "rm_dlu_solve_host": (ctypes.c_int, [_i64, _p, _p, _p, _i64, _p, ctypes.c_int]),
    "rm_dlu_solve_noalloc": (ctypes.c_int, [_i64, _p, _p, _p, _i64, _p, ctypes.c_int, _p]),
    "rm_dsolve": (ctypes.c_int, [_i64, _p, _p, _i64, _p, ctypes.POINTER(SolveOptions), ctypes.POINTER(SolveReport),
                                 _p]),
    "rm_dsolve_host": (ctypes.c_int, [_i64, _p, _p, _i64, _p, ctypes.POINTER(SolveOptions),
                                      ctypes.POINTER(SolveReport)]),
    "rm_batch_plan_create": (ctypes.c_int, [_i64, _p, _p, _p, _p, _p, ctypes.POINTER(SolveOptions),
                                            ctypes.POINTER(_p)]),
    "rm_batch_plan_tune": (ctypes.c_int, [_p, _p, _p, _p, _p]),
    "rm_batch_plan_tune_precision": (ctypes.c_int, [_p, _p, _p, _p, _p]),
    "rm_batch_plan_execute": (ctypes.c_int, [_p, _p, _p, _p, _p]),
    "rm_batch_plan_results": (ctypes.c_int, [_p, _p, _p, _p, ctypes.POINTER(BatchReport)]),
    "rm_batch_plan_panel_width": (ctypes.c_int, [_p, ctypes.c_int]),
    "rm_batch_plan_cta_threads": (ctypes.c_int, [_p, ctypes.c_int]),
    "rm_batch_plan_precision": (ctypes.c_int, [_p, ctypes.c_int]),
    "rm_batch_plan_execute_host": (ctypes.c_int, [_p, _p, _p, _p, _p, _p, _p, _p]),
    "rm_batch_plan_adjoint": (ctypes.c_int, [_p, _p, _p, _p, _p, _p, _p]),
    "rm_dtrsm": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _i64, _i64, _p, _i64, _p,
                                _i64, _p]),
    "rm_dtrsm_host": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _i64, _i64, _p, _i64,
                                     _p, _i64]),
    "rm_dgemm_ozaki_host": (ctypes.c_int, [_i64, _i64, _i64, _p, _i64, _p, _i64, _p, _i64, ctypes.c_int]),
    "rm_dsolve_batched_host": (ctypes.c_int, [_i64, _p, _p, _p, _p, _p, _p, _p, _p, ctypes.POINTER(SolveOptions),
                                              ctypes.POINTER(BatchReport)]),
    "rm_dgemm_ozaki": (ctypes.c_int, [_i64, _i64, _i64, _p, _i64, _p, _i64, _p, _i64, ctypes.c_int, _p]),
    "rm_batch_plan_adjoint_results": (ctypes.c_int, [_p, _p, _p]),
    "rm_batch_plan_destroy": (ctypes.c_int, [_p]),
    "rm_dlu_factor_batched": (ctypes.c_int, [_i64, _i64, _p, _p, _p, _p, _p]),
    "rm_dlu_inverse": (ctypes.c_int, [_i64, _p, _p, _p, _p]),
    "rm_dlu_inverse_host": (ctypes.c_int, [_i64, _p, _p, _p]),
    "rm_dlu_determinant": (ctypes.c_int, [_i64, _i64, _p, _p, _p, _p, _p, _p]),
    "rm_dlu_solve_batched": (ctypes.c_int, [_i64, _i64, _p, _p, _p, _i64, _p, ctypes.c_int, _p]),
    "rm_dcholesky": (ctypes.c_int, [_i64, _p, _p, _p]),
    "rm_dcholesky_host": (ctypes.c_int, [_i64, _p, _p]),
    "rm_dcholesky_batched": (ctypes.c_int, [_i64, _i64, _p, _p, _p, _p]),
    "rm_dcholesky_solve": (ctypes.c_int, [_i64, _p, _p, _i64, _p, _p]),
    "rm_dsolve_batched": (ctypes.c_int, [_i64, _p, _p, _p, _p, _p, _p, _p, _p, ctypes.POINTER(SolveOptions),
                                         ctypes.POINTER(BatchReport), _p]),
}


class RmError(RuntimeError):
    """A failed call into librm_cuda.so, with its status code."""

    def __init__(self, status, message):
        super().__init__(message)
        self.status = status


class NotPositiveDefinite(ValueError):
    """A Cholesky pivot is not > 0: rustymath's cholesky gives None here (and its stacks NaN)."""


class NotRegular(ValueError):
    """A pivot is at most eps*n*max|a|: rustymath's solve would take its least-squares route,
    which this library does not provide."""


_lib = None


def load():
    """The loaded library (built in-tree by rustymath_b200.build); raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: run `python -m rustymath_b200.build` (nvcc, sm_100a)")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype, fn.argtypes = res, args
    _lib = lib
    return lib


def last_error():
    buf = ctypes.create_string_buffer(512)
    load().rm_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(status, what):
    if status == RM_OK:
        return
    text = load().rm_status_string(status).decode()
    detail = last_error()
    msg = f"{what}: {text}" + (f" ({detail})" if detail else "")
    if status == RM_BAD_ARG:
        raise ValueError(msg)
    if status == RM_NOT_REGULAR:
        raise NotRegular(msg)
    if status == RM_NOT_POSITIVE_DEFINITE:
        raise NotPositiveDefinite(msg)
    raise RmError(status, msg)
