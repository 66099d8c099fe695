"""rustymath's dense linear algebra on the B200: `solve`, `lu` (-> `Lu`), `lu_solve`, `det`,
`slogdet`, `cholesky` and `matmul`.

The names, argument meaning, result layouts and errors follow rustymath's Python API
(python/rustymath/linalg.py:26-60 and py/src/linalg.rs:29-107, 226-247):
  - `solve(a, b)`: a is a stack of n x n matrices in its last two axes; a one-dimensional b
    is a vector, otherwise b's last two axes are n x k matrix cells. Frames pair from the
    front, as rustymath broadcasts (tests/test_linalg.py:102-104).
  - `lu(a)` returns `Lu(factors, p)`: factors in rustymath's order, where row j holds column
    j, and p (int64) with row i of L U equal to row p[i] of a. `Lu.solve`, `.inverse`,
    `.determinant`, `.log_determinant`, `.l`, `.u` as in the reference.
  - `det(a)`, `slogdet(a)`: through the LU, as Stacked::det and slogdet
    (src/linalg/stacked.rs:136-171).
  - `cholesky(a)`: L with L L^T = a from a's lower triangle; NaN in every item of a matrix that
    is not positive definite (src/linalg/stacked.rs:259-268).
  - `matmul(a, b)`: the float64 matrix product over frames.
A stack of matrices of order up to 256 goes to the GPU in one launch (batched factorizations
and solves); larger matrices go one at a time through the blocked kernels.

Dtypes follow rustymath's ladder (python/rustymath/linalg.py:1, src/linalg/stacked.rs:76-85,
core/src/buffer.rs:294-315): float64 and float32 results keep their dtype, float16 results
are float16, Booleans and integers up to 16 bits give float32 and wider integers float64 (the
width set by the first argument's dtype, as rustymath's numpy_float policy). The arithmetic
itself is float64 on the GPU throughout: a float32 or float16 result is the float64 result
rounded, at least as accurate as rustymath's float32 computation. Complex matrices are outside
this library.

Arrays may be NumPy arrays (host memory: the call copies to the GPU and back) or torch CUDA
tensors (device memory: the call runs on the current stream). A matrix whose LU pivot is
negligible (rustymath's `regular` test fails) raises NotRegular where rustymath would return
a least-squares solution, which this library does not compute.
"""
import ctypes
from typing import NamedTuple

import numpy as np

from . import _lib
from ._lib import NotRegular, SolveOptions, SolveReport, check

__all__ = ["solve", "lu", "Lu", "lu_solve", "det", "slogdet", "cholesky", "matmul", "matmul_ozaki",
           "NotRegular", "SolveReport", "solve_report"]

_METHODS = {"plain": _lib.RM_METHOD_PLAIN_F64, "f32": _lib.RM_METHOD_F32_IR, "mixed": _lib.RM_METHOD_F32_IR}
BATCH_MAX_N = 256      # the one-launch stack forms take matrices of this order at most
BATCH_MAX_K = 8        # right-hand-side columns per system of the batched solve
SOLVE_BATCH_MAX_K = 64  # right-hand-side columns of the batched solve with given factors
CHOL_BATCH_MAX_N = 128


def _is_torch(x):
    return type(x).__module__.startswith("torch")


def _torch():
    import torch
    return torch


# ---------------------------------------------------------------- dtypes

def _np_dtype(x):
    if _is_torch(x):
        torch = _torch()
        return {torch.float64: np.dtype(np.float64), torch.float32: np.dtype(np.float32),
                torch.float16: np.dtype(np.float16), torch.bfloat16: np.dtype(np.float32),
                torch.bool: np.dtype(np.bool_), torch.uint8: np.dtype(np.uint8), torch.int8: np.dtype(np.int8),
                torch.int16: np.dtype(np.int16), torch.int32: np.dtype(np.int32),
                torch.int64: np.dtype(np.int64)}.get(x.dtype, np.dtype(np.complex128) if x.is_complex() else
                                                     np.dtype(np.float64))
    return np.asarray(x).dtype


def _store_dtype(*xs):
    """The dtype rustymath gives results of these arguments at (stacked.rs:76-85): the widest
    float among them; with no float, the float of the first argument's width policy."""
    dts = [_np_dtype(x) for x in xs]
    if any(d.kind == "c" for d in dts):
        raise TypeError("complex matrices are outside this library (float64 kernels only)")
    if any(d.kind not in "biuf" for d in dts):
        raise TypeError("linalg takes numbers")
    floats = [d for d in dts if d.kind == "f"]
    if floats:
        return max(floats, key=lambda d: d.itemsize)
    first = dts[0]
    return np.dtype(np.float32) if first.kind == "b" or first.itemsize <= 2 else np.dtype(np.float64)


def _torch_dtype(d):
    torch = _torch()
    return {np.dtype(np.float64): torch.float64, np.dtype(np.float32): torch.float32,
            np.dtype(np.float16): torch.float16, np.dtype(np.int64): torch.int64}[np.dtype(d)]


_devices = None


def _require_device():
    """Raises RmError(RM_NO_DEVICE) unless the library sees a compute capability 10.x GPU: the
    functions here never compute anywhere else."""
    global _devices
    if _devices is None:
        c = ctypes.c_int(0)
        _lib.load().rm_device_count(ctypes.byref(c))
        _devices = c.value
    if _devices == 0:
        raise _lib.RmError(_lib.RM_NO_DEVICE, "no compute capability 10.x (B200) device: this library has no CPU path")


def _dev(x):
    """x as a contiguous float64 CUDA tensor (a copy when it is on the host or of another dtype)."""
    _require_device()
    torch = _torch()
    if _is_torch(x):
        t = x.detach()
        if not t.is_cuda:
            t = t.to("cuda")
        return t.to(torch.float64).contiguous()
    return torch.as_tensor(np.ascontiguousarray(np.asarray(x), dtype=np.float64), device="cuda")


def _give(t, like, store):
    """The float64 CUDA result t in the caller's kind (torch CUDA tensor or NumPy array) and
    rustymath's result dtype."""
    if _is_torch(like) and like.is_cuda:
        return t.to(_torch_dtype(store))
    out = t.cpu().numpy().astype(store, copy=False)
    if _is_torch(like):
        return _torch().as_tensor(out)
    return out


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None and t.numel() else None


def _stream():
    return ctypes.c_void_p(_torch().cuda.current_stream().cuda_stream)


def _options(method, max_iterations=30, tolerance=0.0, fallback=True, gmres_restart=20):
    o = SolveOptions()
    o.method = _METHODS[method]
    o.max_iterations = max_iterations
    o.gmres_restart = gmres_restart
    o.fallback = 1 if fallback else 0
    o.tolerance = tolerance
    return o


def _status():
    """Errors the asynchronous kernels recorded (synchronises the current stream)."""
    check(_lib.load().rm_take_status(_stream()), "kernels")


# ---------------------------------------------------------------- solve

def _solve_one(a, b, method, report):
    """One n x n system (float64 CUDA, contiguous) with n x k right-hand sides."""
    torch = _torch()
    n, k = a.shape[-1], b.shape[-1]
    x = torch.empty((n, k), dtype=torch.float64, device=a.device)
    rep = SolveReport()
    opts = _options(method)
    st = _lib.load().rm_dsolve(n, _ptr(a), _ptr(b), k, _ptr(x), ctypes.byref(opts), ctypes.byref(rep), _stream())
    check(st, "solve")
    if report is not None:
        report.append(rep)
    return x


def _solve_stack(a, b, method):
    """count systems of one order n <= BATCH_MAX_N in one batched launch per group of up to
    BATCH_MAX_K right-hand-side columns: a (count, n, n), b (count, n, k), float64 CUDA."""
    torch = _torch()
    count, n, _ = a.shape
    k = b.shape[-1]
    x = torch.empty_like(b)
    lib = _lib.load()
    opts = _options(method)
    ns = np.full(count, n, np.int64)
    a_off = np.arange(count, dtype=np.int64) * n * n
    for c0 in range(0, k, BATCH_MAX_K):
        kc = min(BATCH_MAX_K, k - c0)
        bc = b[..., c0:c0 + kc].contiguous()
        xc = torch.empty_like(bc)
        ks = np.full(count, kc, np.int64)
        b_off = np.arange(count, dtype=np.int64) * n * kc
        rep = _lib.BatchReport()
        st = lib.rm_dsolve_batched(count, ns.ctypes.data, ks.ctypes.data, a_off.ctypes.data, b_off.ctypes.data,
                                   b_off.ctypes.data, _ptr(a), _ptr(bc), _ptr(xc), ctypes.byref(opts),
                                   ctypes.byref(rep), _stream())
        check(st, "solve")
        if rep.not_regular:
            raise NotRegular(f"solve: {rep.not_regular} of the stack's matrices have a pivot at most eps*n*max|a|; "
                             "rustymath's solve takes least squares there")
        x[..., c0:c0 + kc] = xc
    return x


def _frames(a, b):
    """(a frame shape, b frame shape, n, k, vector) with rustymath's pairing rules."""
    if a.ndim < 2:
        raise ValueError("solve needs matrices, with at least two axes")
    m, n = a.shape[-2:]
    if m != n:
        raise ValueError(f"solve needs square matrices, not {m} by {n}")
    if b.ndim == 0:
        raise ValueError("solve needs a right-hand side with at least one axis")
    vector = b.ndim == 1
    rows = b.shape[-1] if vector else b.shape[-2]
    if rows != n:
        raise ValueError(f"solve's right-hand side has {rows} rows, not {n}")
    fa = tuple(a.shape[:-2])
    fb = () if vector else tuple(b.shape[:-2])
    # frames pair from the front: one frame must lead the other
    if fb[:len(fa)] != fa and fa[:len(fb)] != fb:
        raise ValueError(f"solve's frames {fa} and {fb} don't agree")
    return fa, fb, n, (1 if vector else b.shape[-1]), vector


def _shape(x):
    return tuple(x.shape)


def solve(a, b, method="plain", report=None):
    """x with a x = b for each matrix of the stack a (rustymath's `linalg.solve`).

    method "plain" is the float64 LU (the drop-in); "f32"/"mixed" factors in float32 with
    tensor-core updates and refines in float64 to the same backward error. When `report` is
    a list, each system's SolveReport (backward error, iterations, method used) is appended
    (the systems then go one at a time)."""
    like, store = a, _store_dtype(a, b)
    A, B = _dev(a), _dev(b)
    fa, fb, n, k, vector = _frames(A, B)
    if vector:
        B = B.reshape(n, 1)
    lead = fa if len(fa) >= len(fb) else fb
    out_shape = tuple(lead) + ((n,) if vector else (n, k))
    ac = A.reshape(-1, n, n)
    if len(fa) >= len(fb):
        # b's frame leads a's: each b cell pairs with the a cells it prefixes
        extra = fa[len(fb):]
        e = int(np.prod(extra)) if extra else 1
        bc = B.reshape(-1, n, k)
        rhs = bc.repeat_interleave(e, dim=0) if bc.shape[0] > 1 else bc.expand(ac.shape[0], n, k)
        cols = k
    else:
        # a's frame leads b's: all of a cell's right-hand sides solve together, side by side
        extra = fb[len(fa):]
        e = int(np.prod(extra))
        rhs = B.reshape(ac.shape[0], e, n, k).permute(0, 2, 1, 3).reshape(ac.shape[0], n, e * k)
        cols = e * k
    rhs = rhs.contiguous()
    count = ac.shape[0]
    if count > 1 and n <= BATCH_MAX_N and report is None and count * n:
        x = _solve_stack(ac.contiguous(), rhs, method)
    else:
        x = _torch().stack([_solve_one(ac[i].contiguous(), rhs[i].contiguous(), method, report)
                            for i in range(count)]) if count * n else rhs.clone()
    if len(fa) < len(fb):
        x = x.reshape(count, n, e, k).permute(0, 2, 1, 3)
    return _give(x.reshape(out_shape), like, store)


def solve_report(a, b, method="plain"):
    """(x, [SolveReport]) for `solve(a, b, method)`."""
    reps = []
    x = solve(a, b, method=method, report=reps)
    return x, reps


# ---------------------------------------------------------------- LU

class Lu(NamedTuple):
    "Packed LU factors in rustymath's order, where row `j` holds column `j`, and row positions. `l` and `u` give the separate triangular matrices"
    factors: object
    p: object

    @property
    def l(self):
        f = self.factors
        n = f.shape[-1]
        if _is_torch(f):
            torch = _torch()
            t = f.transpose(-1, -2)
            return torch.tril(t, -1) + torch.eye(n, dtype=t.dtype, device=t.device)
        return (np.tril(f.swapaxes(-1, -2), -1) + np.eye(n)).astype(f.dtype)

    @property
    def u(self):
        f = self.factors
        if _is_torch(f):
            return _torch().triu(f.transpose(-1, -2))
        return np.triu(f.swapaxes(-1, -2))

    def solve(self, b):
        "Solve for `b` using these factors, without factoring again or applying a cutoff"
        return lu_solve(self.factors, self.p, b)

    def inverse(self):
        "The inverse from these factors, without factoring again"
        return lu_inverse(self.factors, self.p)

    def determinant(self):
        "The determinant from these factors"
        return _lu_det(self.factors, self.p)[0]

    def log_determinant(self):
        "The determinant's sign and the natural logarithm of its magnitude, from these factors"
        _, sign, log = _lu_det(self.factors, self.p)
        return sign, log


def _lu_cells(A):
    """(factors, perm) of the float64 CUDA stack A (count, n, n): one batched launch for a stack
    of order <= BATCH_MAX_N, the blocked factorization one matrix at a time otherwise."""
    torch = _torch()
    count, n, _ = A.shape
    F = torch.empty_like(A)
    P = torch.empty((count, n), dtype=torch.int64, device=A.device)
    lib = _lib.load()
    if count == 0 or n == 0:
        return F, P
    if count > 1 and n <= BATCH_MAX_N:
        check(lib.rm_dlu_factor_batched(count, n, _ptr(A), _ptr(F), _ptr(P), None, _stream()), "lu")
    else:
        for i in range(count):
            check(lib.rm_dlu_factor(n, _ptr(A[i]), _ptr(F[i]), _ptr(P[i]), None, _stream()), "lu")
    return F, P


def lu(a):
    """The LU factorization with partial pivoting of each matrix of the stack a."""
    like, store = a, _store_dtype(a)
    A = _dev(a)
    if A.ndim < 2 or A.shape[-1] != A.shape[-2]:
        raise ValueError("lu needs square matrices")
    n = A.shape[-1]
    F, P = _lu_cells(A.reshape(-1, n, n).contiguous())
    f = _give(F.reshape(A.shape), like, store)
    if _is_torch(like) and like.is_cuda:
        p = P.reshape(A.shape[:-1])
    else:
        p = P.reshape(A.shape[:-1]).cpu().numpy()
        if _is_torch(like):
            p = _torch().as_tensor(p)
    return Lu(f, p)


def _positions(p, n, shape):
    torch = _torch()
    t = p.detach().to("cuda") if _is_torch(p) else torch.as_tensor(np.asarray(p), device="cuda")
    t = t.to(torch.int64).contiguous()
    if tuple(t.shape) != tuple(shape):
        raise ValueError(f"row positions of shape {tuple(t.shape)} don't match factors of shape {tuple(shape) + (n,)}")
    if t.numel() and bool(((t < 0) | (t >= n)).any().item()):
        raise IndexError(f"lu_solve needs row positions from 0 to {max(n - 1, 0)}")
    return t


def lu_solve(factors, p, b, trans=False):
    """x with a x = b (or a^T x = b when trans) for each matrix that `factors`, `p` describe."""
    torch = _torch()
    like, store = b, _store_dtype(factors, b)
    F, B = _dev(factors), _dev(b)
    n = F.shape[-1]
    fa = tuple(F.shape[:-2])
    P = _positions(p, n, fa + (n,))
    vector = B.ndim == 1
    B2 = B.reshape(n, 1) if vector else B
    if B2.shape[-2] != n:
        raise ValueError(f"lu_solve's right-hand side has {B2.shape[-2]} rows, not {n}")
    k = B2.shape[-1]
    count = int(np.prod(fa)) if fa else 1
    Fc = F.reshape(count, n, n)
    Pc = P.reshape(count, n)
    fb = tuple(B2.shape[:-2])
    if fb not in ((), fa):
        raise ValueError(f"lu_solve's frames {fa} and {fb} don't agree")
    Bc = (B2.reshape(1, n, k).expand(count, n, k) if fb == () else B2.reshape(count, n, k)).contiguous()
    X = torch.empty_like(Bc)
    lib = _lib.load()
    if count * n * k:
        if count > 1 and n <= BATCH_MAX_N and k <= SOLVE_BATCH_MAX_K:
            check(lib.rm_dlu_solve_batched(count, n, _ptr(Fc), _ptr(Pc), _ptr(Bc), k, _ptr(X), int(trans), _stream()),
                  "lu_solve")
        else:
            for i in range(count):
                check(lib.rm_dlu_solve(n, _ptr(Fc[i]), _ptr(Pc[i]), _ptr(Bc[i]), k, _ptr(X[i]), int(trans),
                                       _stream()), "lu_solve")
        _status()
    out = X.reshape(fa + ((n,) if vector else (n, k)))
    return _give(out, like, store)


def lu_inverse(factors, p):
    """The inverse of each matrix that `factors`, `p` describe (rustymath's lu_inverse)."""
    torch = _torch()
    like, store = factors, _store_dtype(factors)
    F = _dev(factors)
    n = F.shape[-1]
    fa = tuple(F.shape[:-2])
    P = _positions(p, n, fa + (n,))
    count = int(np.prod(fa)) if fa else 1
    Fc, Pc = F.reshape(count, n, n), P.reshape(count, n)
    X = torch.empty_like(Fc)
    lib = _lib.load()
    if count * n:
        if count > 1 and n <= min(BATCH_MAX_N, SOLVE_BATCH_MAX_K):
            eye = torch.eye(n, dtype=torch.float64, device=F.device).expand(count, n, n).contiguous()
            check(lib.rm_dlu_solve_batched(count, n, _ptr(Fc), _ptr(Pc), _ptr(eye), n, _ptr(X), 0, _stream()),
                  "inverse")
        else:
            for i in range(count):
                check(lib.rm_dlu_inverse(n, _ptr(Fc[i]), _ptr(Pc[i]), _ptr(X[i]), _stream()), "inverse")
        _status()
    return _give(X.reshape(F.shape), like, store)


def _scalar_or(t, like, store):
    """A rank-0 result as a Python float for host callers (rustymath gives scalars there)."""
    out = _give(t, like, store)
    if not _is_torch(out) and np.ndim(out) == 0:
        return float(out)
    return out


def _lu_det(factors, p):
    """(det, sign, log|det|) of each factorization, folded on the device (rm_dlu_determinant)."""
    torch = _torch()
    like, store = factors, _store_dtype(factors)
    F = _dev(factors)
    n = F.shape[-1]
    fa = tuple(F.shape[:-2])
    P = _positions(p, n, fa + (n,))
    count = int(np.prod(fa)) if fa else 1
    out = torch.empty((3, count), dtype=torch.float64, device=F.device)
    check(_lib.load().rm_dlu_determinant(count, n, _ptr(F), _ptr(P), _ptr(out[0]), _ptr(out[1]), _ptr(out[2]),
                                         _stream()), "determinant")
    _status()
    return tuple(_scalar_or(out[i].reshape(fa), like, store) for i in range(3))


def det(a):
    """The determinant of each matrix of the stack a, through its LU (Stacked::det)."""
    f = lu(a)
    return _lu_det(f.factors, f.p)[0]


def slogdet(a):
    """(sign, log|det|) of each matrix of the stack a, through its LU (Stacked::slogdet)."""
    f = lu(a)
    _, sign, log = _lu_det(f.factors, f.p)
    return sign, log


# ---------------------------------------------------------------- Cholesky

def cholesky(a):
    """L with L L^T = a for each symmetric positive definite matrix of the stack a, reading only
    its lower triangle; NaN in every item of a matrix that is not positive definite, as
    rustymath's stacks give (src/linalg/stacked.rs:259-268)."""
    torch = _torch()
    like, store = a, _store_dtype(a)
    A = _dev(a)
    if A.ndim < 2 or A.shape[-1] != A.shape[-2]:
        raise ValueError("cholesky needs square matrices")
    n = A.shape[-1]
    Ac = A.reshape(-1, n, n).contiguous()
    count = Ac.shape[0]
    L = torch.empty_like(Ac)
    lib = _lib.load()
    if count * n:
        if n <= CHOL_BATCH_MAX_N:
            check(lib.rm_dcholesky_batched(count, n, _ptr(Ac), _ptr(L), None, _stream()), "cholesky")
            _status()
        else:
            for i in range(count):
                st = lib.rm_dcholesky(n, _ptr(Ac[i]), _ptr(L[i]), _stream())
                if st == _lib.RM_NOT_POSITIVE_DEFINITE:
                    L[i] = float("nan")
                else:
                    check(st, "cholesky")
    return _give(L.reshape(A.shape), like, store)


# ---------------------------------------------------------------- products

def _as_f64(x):
    if _is_torch(x):
        torch = _torch()
        if not x.is_cuda:
            return np.ascontiguousarray(x.detach().cpu().numpy(), dtype=np.float64), False
        return x.detach().to(torch.float64).contiguous(), True
    return np.ascontiguousarray(np.asarray(x), dtype=np.float64), False


def _hptr(x, device):
    if device:
        return ctypes.c_void_p(x.data_ptr())
    return ctypes.c_void_p(x.ctypes.data) if x.size else None


def _empty(shape, like, device):
    if device:
        torch = _torch()
        return torch.empty(shape, dtype=torch.float64, device=like.device)
    return np.empty(shape, dtype=np.float64)


def _contig(x, device):
    return x.contiguous() if device else np.ascontiguousarray(x)


def _stack(xs, device):
    if device:
        return _torch().stack(xs)
    return np.stack(xs)


def matmul(a, b):
    """The float64 matrix product a @ b (rustymath's `matmul` for float64 matrices)."""
    a, dev_a = _as_f64(a)
    b, dev_b = _as_f64(b)
    if dev_a != dev_b:
        raise ValueError("matmul's arguments must both be on the GPU or both on the host")
    device = dev_a
    va, vb = a.ndim == 1, b.ndim == 1
    a2 = a.reshape(1, -1) if va else a
    b2 = b.reshape(-1, 1) if vb else b
    if a2.ndim != 2 or b2.ndim != 2:
        return _matmul_frames(a2, b2, device, va, vb)
    m, k = a2.shape
    k2, n = b2.shape
    if k != k2:
        raise ValueError(f"matmul contracts {k} with {k2} items")
    c = _gemm(_contig(a2, device), _contig(b2, device), device)
    if va and vb:
        return c.reshape(())[()] if not device else c.reshape(())
    if va:
        return c.reshape(n)
    if vb:
        return c.reshape(m)
    return c


def matmul_ozaki(a, b, slices=8):
    """a @ b for float64 CUDA matrices from int8 tensor-core products (rm_dgemm_ozaki): rows of
    a and columns of b cut into `slices` 7-bit pieces; 8 slices give float64-level accuracy."""
    torch = _torch()
    if not (_is_torch(a) and _is_torch(b) and a.is_cuda and b.is_cuda):
        raise ValueError("matmul_ozaki works on CUDA tensors")
    a = a.to(torch.float64).contiguous()
    b = b.to(torch.float64).contiguous()
    if a.ndim != 2 or b.ndim != 2 or a.shape[1] != b.shape[0]:
        raise ValueError("matmul_ozaki needs an m x k and a k x n matrix")
    m, k = a.shape
    n = b.shape[1]
    c = torch.empty((m, n), dtype=torch.float64, device=a.device)
    if m and n:
        st = _lib.load().rm_dgemm_ozaki(m, n, k, _hptr(a, True), max(k, 1), _hptr(b, True), max(n, 1), _hptr(c, True),
                                        n, slices, _stream())
        check(st, "matmul_ozaki")
    return c


def _gemm(a, b, device):
    m, k = a.shape
    n = b.shape[1]
    c = _empty((m, n), a, device)
    if device and m * n:
        c.zero_()
    elif m * n:
        c.fill(0.0)
    if m and n:
        lib = _lib.load()
        if device:
            st = lib.rm_dgemm(0, 0, m, n, k, 1.0, _hptr(a, True), max(k, 1), _hptr(b, True), max(n, 1), 0.0,
                              _hptr(c, True), n, _stream())
        else:
            st = lib.rm_dgemm_host(0, 0, m, n, k, 1.0, _hptr(a, False), max(k, 1), _hptr(b, False), max(n, 1), 0.0,
                                   _hptr(c, False), n)
        check(st, "matmul")
    return c


def _matmul_frames(a, b, device, va, vb):
    fa, fb = a.shape[:-2], b.shape[:-2]
    if fb[:len(fa)] != fa and fa[:len(fb)] != fb:
        raise ValueError(f"matmul's frames {fa} and {fb} don't agree")
    lead = fa if len(fa) >= len(fb) else fb
    count = int(np.prod(lead))
    ea = int(np.prod(lead[len(fa):])) if len(lead) > len(fa) else 1
    eb = int(np.prod(lead[len(fb):])) if len(lead) > len(fb) else 1
    ac = a.reshape((-1,) + a.shape[-2:])
    bc = b.reshape((-1,) + b.shape[-2:])
    cells = [_gemm(_contig(ac[i // ea], device), _contig(bc[i // eb], device), device) for i in range(count)]
    out = _stack(cells, device)
    shape = tuple(lead) + out.shape[-2:]
    out = out.reshape(shape)
    if va:
        out = out.reshape(shape[:-2] + (shape[-1],))
    if vb:
        out = out.reshape(shape[:-1])
    return out
