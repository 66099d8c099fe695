"""ctypes binding of the CPU oracle (oracle/rm_oracle.c).

Test infrastructure only: tests/, the smoke check and bench.py's CPU-baseline leg import
this module as the checker and as the timed CPU baseline. The product path never imports
it. The library restates rustymath's dense f64 algorithms (see rm_oracle.c's header for the
reference files it follows)."""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")

_i64, _f64, _p = ctypes.c_int64, ctypes.c_double, ctypes.c_void_p


def build():
    """Compiles liboracle.so from rm_oracle.c with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def _load():
    if not os.path.exists(LIB):
        build()
    lib = ctypes.CDLL(LIB)
    sig = {
        "ora_set_threads": (None, [ctypes.c_int]),
        "ora_get_threads": (ctypes.c_int, []),
        "ora_dgemm": (None, [ctypes.c_int, ctypes.c_int, _i64, _i64, _i64, _f64, _p, _i64, _p, _i64, _f64, _p, _i64]),
        "ora_dgemm_fold": (None, [_i64, _i64, _i64, _f64, _p, _p, _f64, _p]),
        "ora_lu_factor": (None, [_i64, _p, _p, _p]),
        "ora_lu_factor_pivots": (None, [_i64, _p, _p, _p]),
        "ora_lu_solve": (None, [_i64, _p, _p, _p, _i64, _p]),
        "ora_lu_solve_transposed": (None, [_i64, _p, _p, _p, _i64, _p]),
        "ora_lu_inverse": (None, [_i64, _p, _p, _p]),
        "ora_lu_determinant": (_f64, [_i64, _p, _p]),
        "ora_lu_log_determinant": (None, [_i64, _p, _p, _p, _p]),
        "ora_regular": (ctypes.c_int, [_i64, _p, _p]),
        "ora_cholesky": (ctypes.c_int, [_i64, _p, _p]),
        "ora_solve": (ctypes.c_int, [_i64, _p, _p, _i64, _p]),
        "ora_backward_error": (_f64, [_i64, _p, _p, _p, _i64]),
        "ora_residual_dd": (None, [_i64, _p, _p, _p, _i64, _p]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype, f.argtypes = res, args
    return lib


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = _load()
    return _lib


def _c(x, dtype=np.float64):
    return np.ascontiguousarray(x, dtype=dtype)


def _ptr(x):
    return x.ctypes.data if x.size else None


def set_threads(t):
    lib().ora_set_threads(int(t))


def get_threads():
    return lib().ora_get_threads()


def dgemm(a, b, alpha=1.0, beta=0.0, c=None, ta=False, tb=False):
    """C = alpha*op(A)*op(B) + beta*C for row-major float64 arrays."""
    a, b = _c(a), _c(b)
    m, k = (a.shape[1], a.shape[0]) if ta else a.shape
    kb, n = (b.shape[1], b.shape[0]) if tb else b.shape
    assert k == kb
    out = np.zeros((m, n)) if c is None else _c(c).copy()
    lib().ora_dgemm(int(ta), int(tb), m, n, k, alpha, _ptr(a), a.shape[1] if a.size else 1,
                    _ptr(b), b.shape[1] if b.size else 1, beta, _ptr(out), max(n, 1))
    return out


def dgemm_fold(a, b, alpha=1.0, beta=0.0, c=None):
    a, b = _c(a), _c(b)
    m, k = a.shape
    n = b.shape[1]
    out = np.zeros((m, n)) if c is None else _c(c).copy()
    lib().ora_dgemm_fold(m, n, k, alpha, _ptr(a), _ptr(b), beta, _ptr(out))
    return out


def lu_factor(a):
    """(factors column-major as an n*n array where row j holds column j, perm int64)."""
    a = _c(a)
    n = a.shape[0]
    f = np.zeros((n, n))
    p = np.zeros(n, np.int64)
    lib().ora_lu_factor(n, _ptr(a), _ptr(f), _ptr(p))
    return f, p


def lu_pivots(a):
    a = _c(a)
    n = a.shape[0]
    f = np.zeros((n, n))
    piv = np.zeros(n, np.int64)
    lib().ora_lu_factor_pivots(n, _ptr(a), _ptr(f), _ptr(piv))
    return f, piv


def _rhs(b):
    b = _c(b)
    vector = b.ndim == 1
    return (b.reshape(-1, 1) if vector else b), vector


def lu_solve(factors, perm, b):
    f, p = _c(factors), _c(perm, np.int64)
    b2, vector = _rhs(b)
    n, k = b2.shape
    x = np.zeros((n, k))
    lib().ora_lu_solve(n, _ptr(f), _ptr(p), _ptr(b2), k, _ptr(x))
    return x[:, 0] if vector else x


def lu_solve_transposed(factors, perm, b):
    f, p = _c(factors), _c(perm, np.int64)
    b2, vector = _rhs(b)
    n, k = b2.shape
    x = np.zeros((n, k))
    lib().ora_lu_solve_transposed(n, _ptr(f), _ptr(p), _ptr(b2), k, _ptr(x))
    return x[:, 0] if vector else x


def lu_inverse(factors, perm):
    f, p = _c(factors), _c(perm, np.int64)
    n = f.shape[0]
    out = np.zeros((n, n))
    lib().ora_lu_inverse(n, _ptr(f), _ptr(p), _ptr(out))
    return out


def lu_determinant(factors, perm):
    f, p = _c(factors), _c(perm, np.int64)
    return lib().ora_lu_determinant(f.shape[0], _ptr(f), _ptr(p))


def lu_log_determinant(factors, perm):
    f, p = _c(factors), _c(perm, np.int64)
    s, l = ctypes.c_double(), ctypes.c_double()
    lib().ora_lu_log_determinant(f.shape[0], _ptr(f), _ptr(p), ctypes.addressof(s), ctypes.addressof(l))
    return s.value, l.value


def cholesky(a):
    """L with L L^T = A (row-major, zeros above the diagonal), or None where A is not positive
    definite: rustymath's cholesky (core/src/linalg/factor.rs:750-795)."""
    a = _c(a)
    n = a.shape[0]
    out = np.zeros((n, n))
    ok = lib().ora_cholesky(n, _ptr(a), _ptr(out))
    return out if ok else None


def regular(a, factors):
    a, f = _c(a), _c(factors)
    return bool(lib().ora_regular(a.shape[0], _ptr(a), _ptr(f)))


def solve(a, b):
    """x for a regular square a, or None where the reference would take lstsq."""
    a = _c(a)
    b2, vector = _rhs(b)
    n, k = b2.shape
    x = np.zeros((n, k))
    status = lib().ora_solve(n, _ptr(a), _ptr(b2), k, _ptr(x))
    if status != 0:
        return None
    return x[:, 0] if vector else x


def backward_error(a, x, b):
    a = _c(a)
    x2, _ = _rhs(x)
    b2, _ = _rhs(b)
    return lib().ora_backward_error(a.shape[0], _ptr(a), _ptr(x2), _ptr(b2), b2.shape[1])


def residual_dd(a, x, b):
    a = _c(a)
    x2, vector = _rhs(x)
    b2, _ = _rhs(b)
    r = np.zeros_like(b2)
    lib().ora_residual_dd(a.shape[0], _ptr(a), _ptr(x2), _ptr(b2), b2.shape[1], _ptr(r))
    return r[:, 0] if vector else r
