"""rustymath's dense float64 linear algebra on the B200: `solve`, `lu` (-> `Lu`) and `matmul`.

The names, argument meaning, result layouts and errors follow rustymath's Python API
(python/rustymath/linalg.py:26-60 and py/src/linalg.rs:29-70, 226-247):
  - `solve(a, b)`: a is a stack of n x n matrices in its last two axes; a one-dimensional b
    is a vector, otherwise b's last two axes are n x k matrix cells. Frames pair from the
    front, as rustymath broadcasts (tests/test_linalg.py:102-104).
  - `lu(a)` returns `Lu(factors, p)`: factors in rustymath's order, where row j holds column
    j, and p (int64) with row i of L U equal to row p[i] of a. `Lu.solve`, `.inverse`,
    `.determinant`, `.log_determinant`, `.l`, `.u` as in the reference.
  - `matmul(a, b)`: the float64 matrix product over frames.
Arrays may be NumPy arrays (host memory: the call copies to the GPU and back) or torch
CUDA tensors (device memory: the call runs on the current stream). Everything computes in
float64 on the GPU through librm_cuda.so; other float and integer dtypes are converted to
float64 and results given at float64. A matrix whose LU pivot is negligible (rustymath's
`regular` test fails) raises NotRegular where rustymath would return a least-squares
solution, which this library does not compute.
"""
import ctypes
from typing import NamedTuple

import numpy as np

from . import _lib
from ._lib import NotRegular, SolveOptions, SolveReport, check

__all__ = ["solve", "lu", "Lu", "matmul", "matmul_ozaki", "lu_solve", "NotRegular", "SolveReport", "solve_report"]

_METHODS = {"plain": _lib.RM_METHOD_PLAIN_F64, "f32": _lib.RM_METHOD_F32_IR, "mixed": _lib.RM_METHOD_F32_IR}


def _is_torch(x):
    return type(x).__module__.startswith("torch")


def _torch():
    import torch
    return torch


def _as_f64(x):
    if _is_torch(x):
        torch = _torch()
        if not x.is_cuda:
            return np.ascontiguousarray(x.detach().cpu().numpy(), dtype=np.float64), False
        return x.detach().to(torch.float64).contiguous(), True
    return np.ascontiguousarray(np.asarray(x), dtype=np.float64), False


def _ptr(x, device):
    if device:
        return ctypes.c_void_p(x.data_ptr())
    return ctypes.c_void_p(x.ctypes.data) if x.size else None


def _stream(device):
    if not device:
        return None
    return ctypes.c_void_p(_torch().cuda.current_stream().cuda_stream)


def _empty(shape, like, device, dtype=np.float64):
    if device:
        torch = _torch()
        tdt = torch.float64 if dtype == np.float64 else torch.int64
        return torch.empty(shape, dtype=tdt, device=like.device)
    return np.empty(shape, dtype=dtype)


def _options(method, max_iterations=30, tolerance=0.0, fallback=True, gmres_restart=20):
    o = SolveOptions()
    o.method = _METHODS[method]
    o.max_iterations = max_iterations
    o.gmres_restart = gmres_restart
    o.fallback = 1 if fallback else 0
    o.tolerance = tolerance
    return o


def _solve_cell(a, b, device, method, report):
    """One n x n system with n x k right-hand sides (both contiguous float64)."""
    n, k = a.shape[-1], b.shape[-1]
    x = _empty((n, k), a, device)
    rep = SolveReport()
    opts = _options(method)
    lib = _lib.load()
    if device:
        st = lib.rm_dsolve(n, _ptr(a, True), _ptr(b, True), k, _ptr(x, True), ctypes.byref(opts), ctypes.byref(rep),
                           _stream(True))
    else:
        st = lib.rm_dsolve_host(n, _ptr(a, False), _ptr(b, False), k, _ptr(x, False), ctypes.byref(opts),
                                ctypes.byref(rep))
    check(st, "solve")
    if report is not None:
        report.append(rep)
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


def solve(a, b, method="plain", report=None):
    """x with a x = b for each matrix of the stack a (rustymath's `linalg.solve`).

    method "plain" is the float64 LU (the drop-in); "f32"/"mixed" factors in float32 with
    tensor-core updates and refines in float64 to the same backward error. When `report` is
    a list, each system's SolveReport (backward error, iterations, method used) is appended."""
    a, dev_a = _as_f64(a)
    b, dev_b = _as_f64(b)
    if dev_a != dev_b:
        raise ValueError("solve's arguments must both be on the GPU or both on the host")
    device = dev_a
    fa, fb, n, k, vector = _frames(a, b)
    if vector:
        b = b.reshape(n, 1)
    lead = fa if len(fa) >= len(fb) else fb
    out_shape = tuple(lead) + ((n,) if vector else (n, k))
    if len(fa) >= len(fb):
        # b's frame leads a's: each b cell pairs with the a cells it prefixes
        extra = fa[len(fb):]
        ac = a.reshape((-1, n, n)) if fa else a.reshape(1, n, n)
        bcells = b.reshape((-1, n, k)) if fb else b.reshape(1, n, k)
        e = int(np.prod(extra)) if extra else 1
        xs = []
        for i in range(ac.shape[0]):
            bi = bcells[i // e] if bcells.shape[0] > 1 else bcells[0]
            xs.append(_solve_cell(ac[i], _contig(bi, device), device, method, report))
    else:
        # a's frame leads b's: all of a cell's right-hand sides solve together
        extra = fb[len(fa):]
        e = int(np.prod(extra))
        ac = a.reshape((-1, n, n)) if fa else a.reshape(1, n, n)
        bc = b.reshape((ac.shape[0], e, n, k))
        xs = []
        for i in range(ac.shape[0]):
            rhs = _cat_columns(bc[i], device)  # n x (e*k)
            x = _solve_cell(ac[i], rhs, device, method, report)
            xs.append(_split_columns(x, e, k, device))
    x = _stack(xs, device).reshape(out_shape)
    return x


def solve_report(a, b, method="plain"):
    """(x, [SolveReport]) for `solve(a, b, method)`."""
    reps = []
    x = solve(a, b, method=method, report=reps)
    return x, reps


def _contig(x, device):
    return x.contiguous() if device else np.ascontiguousarray(x)


def _cat_columns(cells, device):
    # cells: (e, n, k) -> (n, e*k)
    if device:
        return cells.permute(1, 0, 2).reshape(cells.shape[1], -1).contiguous()
    return np.ascontiguousarray(np.transpose(cells, (1, 0, 2)).reshape(cells.shape[1], -1))


def _split_columns(x, e, k, device):
    n = x.shape[0]
    if device:
        return x.reshape(n, e, k).permute(1, 0, 2).contiguous()
    return np.ascontiguousarray(np.transpose(x.reshape(n, e, k), (1, 0, 2)))


def _stack(xs, device):
    if device:
        return _torch().stack(xs)
    return np.stack(xs)


class Lu(NamedTuple):
    "Packed LU factors in rustymath's order, where row `j` holds column `j`, and row positions. `l` and `u` give the separate triangular matrices"
    factors: object
    p: object

    @property
    def l(self):
        f = self.factors
        t = f.swapaxes(-1, -2) if not _is_torch(f) else f.transpose(-1, -2)
        n = f.shape[-1]
        if _is_torch(f):
            torch = _torch()
            return torch.tril(t, -1) + torch.eye(n, dtype=t.dtype, device=t.device)
        return np.tril(t, -1) + np.eye(n)

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
        f = self.factors
        n = f.shape[-1]
        eye = _torch().eye(n, dtype=_torch().float64, device=f.device) if _is_torch(f) else np.eye(n)
        if f.ndim == 2:
            return lu_solve(f, self.p, eye)
        cells = [lu_solve(f[i], self.p[i], eye) for i in range(f.shape[0])]
        return _stack(cells, _is_torch(f))

    def determinant(self):
        "The determinant from these factors: U's diagonal product, negated for an odd p (factor.rs:174-176)"
        f, p = self.factors, self.p
        if _is_torch(f):
            return _torch().prod(_torch().diagonal(f, dim1=-2, dim2=-1), -1) * _parity(p)
        d = np.diagonal(f, axis1=-2, axis2=-1)
        prod = np.ones(d.shape[:-1])
        for i in range(d.shape[-1]):  # in order, as the reference folds it
            prod = prod * d[..., i]
        out = prod * _parity(p)
        return float(out) if np.ndim(out) == 0 else out

    def log_determinant(self):
        "The determinant's sign and the natural logarithm of its magnitude, from these factors"
        return self._signs()

    def _signs(self):
        f, p = self.factors, self.p
        if _is_torch(f):
            torch = _torch()
            d = torch.diagonal(f, dim1=-2, dim2=-1)
            zero = (d == 0).any(-1)
            sign = torch.where(zero, torch.zeros_like(d[..., 0]), torch.prod(torch.sign(d), -1) * _parity(p))
            log = torch.where(zero, torch.full_like(d[..., 0], -float("inf")), torch.log(torch.abs(d)).sum(-1))
            return sign, log
        d = np.diagonal(f, axis1=-2, axis2=-1)
        zero = (d == 0).any(-1)
        with np.errstate(divide="ignore"):
            sign = np.where(zero, 0.0, np.prod(np.sign(d), -1) * _parity(p))
            log = np.where(zero, -np.inf, np.log(np.abs(d)).sum(-1))
        if np.ndim(sign) == 0:
            return float(sign), float(log)
        return sign, log


def _parity(p):
    """+1 / -1 for an even / odd permutation (rustymath's `odd`, factor.rs:186-194)."""
    pn = p.detach().cpu().numpy() if _is_torch(p) else np.asarray(p)
    flat = pn.reshape(-1, pn.shape[-1])
    out = []
    for row in flat:
        n = len(row)
        seen = np.zeros(n, bool)
        cycles = 0
        for s in range(n):
            if not seen[s]:
                cycles += 1
                i = s
                while not seen[i]:
                    seen[i] = True
                    i = int(row[i])
        out.append(-1.0 if (n - cycles) % 2 else 1.0)
    res = np.array(out).reshape(pn.shape[:-1])
    if _is_torch(p):
        return _torch().as_tensor(res, dtype=_torch().float64, device=p.device)
    return res if res.ndim else float(res)


def lu(a):
    """The LU factorization with partial pivoting of each matrix of the stack a."""
    a, device = _as_f64(a)
    if a.ndim < 2 or a.shape[-1] != a.shape[-2]:
        raise ValueError("lu needs square matrices")
    n = a.shape[-1]
    cells = a.reshape(-1, n, n)
    fs, ps = [], []
    lib = _lib.load()
    for i in range(cells.shape[0]):
        ai = _contig(cells[i], device)
        f = _empty((n, n), ai, device)
        p = _empty((n,), ai, device, np.int64)
        if n:
            if device:
                st = lib.rm_dlu_factor(n, _ptr(ai, True), _ptr(f, True), _ptr(p, True), None, _stream(True))
            else:
                st = lib.rm_dlu_factor_host(n, _ptr(ai, False), _ptr(f, False), _ptr(p, False), None)
            check(st, "lu")
        fs.append(f)
        ps.append(p)
    if a.ndim == 2:
        return Lu(fs[0], ps[0])
    return Lu(_stack(fs, device).reshape(a.shape), _stack(ps, device).reshape(a.shape[:-1]))


def _positions(p, n, device):
    if device:
        torch = _torch()
        p = p.to(torch.int64).contiguous()
        bad = ((p < 0) | (p >= n)).any().item()
    else:
        p = np.ascontiguousarray(np.asarray(p), dtype=np.int64)
        bad = bool(((p < 0) | (p >= n)).any())
    if bad:
        raise IndexError(f"lu_solve needs row positions from 0 to {max(n - 1, 0)}")
    return p


def lu_solve(factors, p, b, trans=False):
    """x with a x = b (or a^T x = b when trans) for the matrix that `factors`, `p` describe."""
    f, device = _as_f64(factors)
    b, dev_b = _as_f64(b)
    if device != dev_b:
        raise ValueError("lu_solve's arguments must both be on the GPU or both on the host")
    n = f.shape[-1]
    vector = b.ndim == 1
    b2 = b.reshape(n, 1) if vector else b
    if b2.shape[-2] != n:
        raise ValueError(f"lu_solve's right-hand side has {b2.shape[-2]} rows, not {n}")
    p = _positions(p, n, device)
    k = b2.shape[-1]
    b2 = _contig(b2, device)
    x = _empty((n, k), b2, device)
    lib = _lib.load()
    if n and k:
        if device:
            st = lib.rm_dlu_solve(n, _ptr(f, True), _ptr(p, True), _ptr(b2, True), k, _ptr(x, True), int(trans),
                                  _stream(True))
            if st == _lib.RM_OK:  # errors the kernels found (the device form is asynchronous)
                st = lib.rm_take_status(_stream(True))
        else:
            st = lib.rm_dlu_solve_host(n, _ptr(f, False), _ptr(p, False), _ptr(b2, False), k, _ptr(x, False),
                                       int(trans))
        check(st, "lu_solve")
    return x.reshape(n) if vector else x


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
        st = _lib.load().rm_dgemm_ozaki(m, n, k, _ptr(a, True), max(k, 1), _ptr(b, True), max(n, 1), _ptr(c, True),
                                        n, slices, _stream(True))
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
            st = lib.rm_dgemm(0, 0, m, n, k, 1.0, _ptr(a, True), max(k, 1), _ptr(b, True), max(n, 1), 0.0,
                              _ptr(c, True), n, _stream(True))
        else:
            st = lib.rm_dgemm_host(0, 0, m, n, k, 1.0, _ptr(a, False), max(k, 1), _ptr(b, False), max(n, 1), 0.0,
                                   _ptr(c, False), n)
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
