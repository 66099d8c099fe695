"""Many small systems of uneven size solved in one persistent, graph-replayed launch.

rustymath solves a stack of same-size systems one LuWork per thread (Stacked::solve,
src/linalg/stacked.rs:88-101); `solve_batched` takes systems of different sizes (n <= 256,
k <= 8 right-hand sides each), which a rustymath stack cannot hold, and solves them all in
one kernel launch: float32 LU with partial pivoting and float64 refinement per system
("mixed", falling back to a float64 LU for a system whose refinement stalls) or float64 LU
("plain"). `BatchPlan` keeps the layout, scratch and CUDA graph for repeated solves of the
same shapes, and `tune()` picks the panel width of each size bucket by timing.
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import BatchReport, check
from .linalg import _METHODS, _is_torch, _options, _torch

__all__ = ["BatchPlan", "solve_batched", "BatchReport"]


def _offsets(ns, ks):
    ns = np.asarray(ns, dtype=np.int64)
    ks = np.asarray(ks, dtype=np.int64)
    a_off = np.concatenate([[0], np.cumsum(ns * ns)[:-1]]).astype(np.int64) if len(ns) else np.zeros(0, np.int64)
    b_off = np.concatenate([[0], np.cumsum(ns * ks)[:-1]]).astype(np.int64) if len(ns) else np.zeros(0, np.int64)
    return ns, ks, a_off, b_off, int((ns * ns).sum()), int((ns * ks).sum())


class BatchPlan:
    """The plan for a batch of shapes: systems i has an ns[i] x ns[i] matrix and ns[i] x ks[i]
    right-hand sides, packed back to back (row-major) in flat float64 arrays: `pack` builds
    them, `unpack` splits solutions."""

    def __init__(self, ns, ks, method="mixed", fallback=True, tolerance=0.0, max_iterations=30):
        self.ns, self.ks, self.a_off, self.b_off, self.a_size, self.b_size = _offsets(ns, ks)
        self.count = len(self.ns)
        self._opts = _options(method, max_iterations=max_iterations, tolerance=tolerance, fallback=fallback)
        lib = _lib.load()
        h = ctypes.c_void_p()
        st = lib.rm_batch_plan_create(self.count, self.ns.ctypes.data, self.ks.ctypes.data, self.a_off.ctypes.data,
                                      self.b_off.ctypes.data, self.b_off.ctypes.data, ctypes.byref(self._opts),
                                      ctypes.byref(h))
        check(st, "batch plan")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            _lib.load().rm_batch_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def pack(self, As, Bs, device=None):
        """Flat float64 A and B from lists of matrices (device: a torch device to place them on)."""
        a = np.concatenate([np.ascontiguousarray(x, dtype=np.float64).ravel() for x in As]) if As else np.zeros(0)
        b = np.concatenate([np.ascontiguousarray(np.asarray(x, dtype=np.float64).reshape(n, k)).ravel()
                            for x, n, k in zip(Bs, self.ns, self.ks)]) if Bs else np.zeros(0)
        if device is not None:
            torch = _torch()
            return torch.as_tensor(a, device=device), torch.as_tensor(b, device=device)
        return a, b

    def unpack(self, x):
        """The list of n x k solutions inside the flat x."""
        return [x[o:o + n * k].reshape(n, k) for o, n, k in zip(self.b_off, self.ns, self.ks)]

    def _ptrs(self, a, b, x):
        torch = _torch()
        for t in (a, b, x):
            if not (_is_torch(t) and t.is_cuda and t.dtype == torch.float64 and t.is_contiguous()):
                raise ValueError("BatchPlan works on contiguous float64 CUDA tensors")
        if a.numel() < self.a_size or b.numel() < self.b_size or x.numel() < self.b_size:
            raise ValueError("the packed arrays are smaller than the plan's shapes")
        return (ctypes.c_void_p(a.data_ptr()), ctypes.c_void_p(b.data_ptr()), ctypes.c_void_p(x.data_ptr()),
                ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))

    def tune(self, a, b, x, precision=False):
        """Times the candidate panel widths per size bucket, and the CTA size for the systems of
        n <= 64, on these inputs; keeps the fastest. With `precision` (a mixed plan), each bucket
        also times float64 factors without refinement and keeps the faster route (see
        `precision()`). Returns the panel widths per bucket."""
        fn = _lib.load().rm_batch_plan_tune_precision if precision else _lib.load().rm_batch_plan_tune
        check(fn(self._h, *self._ptrs(a, b, x)), "batch tune")
        return [_lib.load().rm_batch_plan_panel_width(self._h, i) for i in range(5)]

    def precision(self):
        """The route of each size bucket (n <= 32, 64, 128, 192, 256): "mixed" (float32 factors +
        float64 refinement) or "plain" (float64 factors)."""
        names = {_lib.RM_METHOD_PLAIN_F64: "plain", _lib.RM_METHOD_F32_IR: "mixed"}
        return [names.get(_lib.load().rm_batch_plan_precision(self._h, i), "?") for i in range(5)]

    def cta_threads(self):
        """Threads per CTA (a thread per row: 64 or 256) solving each size bucket (n <= 32, 64,
        128, 192, 256)."""
        return [_lib.load().rm_batch_plan_cta_threads(self._h, i) for i in range(5)]

    def execute(self, a, b, x):
        """One persistent launch for every system (asynchronous on the current stream)."""
        check(_lib.load().rm_batch_plan_execute(self._h, *self._ptrs(a, b, x)), "batch execute")

    def execute_host(self, a_h, b_h, x_h, a, b, x):
        """execute from host memory: copies the CPU tensors a_h, b_h (pinned, for the copies to
        overlap the solves) into the CUDA tensors a, b, solves, and copies x back into x_h, group
        by group; asynchronous on the current stream (x_h is complete once it synchronises)."""
        torch = _torch()
        for t in (a_h, b_h, x_h):
            if not (_is_torch(t) and not t.is_cuda and t.dtype == torch.float64 and t.is_contiguous()):
                raise ValueError("execute_host takes contiguous float64 CPU tensors")
        if a_h.numel() < self.a_size or b_h.numel() < self.b_size or x_h.numel() < self.b_size:
            raise ValueError("the packed host arrays are smaller than the plan's shapes")
        pa, pb, px, s = self._ptrs(a, b, x)
        check(_lib.load().rm_batch_plan_execute_host(self._h, ctypes.c_void_p(a_h.data_ptr()),
                                                     ctypes.c_void_p(b_h.data_ptr()), ctypes.c_void_p(x_h.data_ptr()),
                                                     pa, pb, px, s), "batch execute_host")

    def adjoint(self, a, x, gx, gb, ga=None):
        """gb = A^-T gx and (unless ga is None) ga = -gb x^T for every system, from the factors
        of the last execute (a and x must be that execute's); asynchronous."""
        torch = _torch()
        for t in (gx, gb) + (() if ga is None else (ga,)):
            if not (_is_torch(t) and t.is_cuda and t.dtype == torch.float64 and t.is_contiguous()):
                raise ValueError("BatchPlan works on contiguous float64 CUDA tensors")
        if gx.numel() < self.b_size or gb.numel() < self.b_size or (ga is not None and ga.numel() < self.a_size):
            raise ValueError("the packed arrays are smaller than the plan's shapes")
        pa, _, px, ps = self._ptrs(a, gx, x)
        check(_lib.load().rm_batch_plan_adjoint(self._h, pa, px, ctypes.c_void_p(gx.data_ptr()),
                                                ctypes.c_void_p(gb.data_ptr()),
                                                None if ga is None else ctypes.c_void_p(ga.data_ptr()), ps),
              "batch adjoint")

    def adjoint_results(self):
        """(per-system backward errors of A^T gb = gx, their maximum) of the last adjoint."""
        berr = np.zeros(self.count)
        mx = ctypes.c_double()
        check(_lib.load().rm_batch_plan_adjoint_results(self._h, berr.ctypes.data if self.count else None,
                                                        ctypes.byref(mx)), "batch adjoint results")
        return berr, mx.value

    def results(self):
        """(backward errors, refinement steps, RM_BATCH_* flags, BatchReport) of the last execute."""
        berr = np.zeros(self.count)
        iters = np.zeros(self.count, np.int32)
        flags = np.zeros(self.count, np.int32)
        rep = BatchReport()
        check(_lib.load().rm_batch_plan_results(self._h, berr.ctypes.data if self.count else None,
                                                iters.ctypes.data if self.count else None,
                                                flags.ctypes.data if self.count else None, ctypes.byref(rep)),
              "batch results")
        return berr, iters, flags, rep


def solve_batched(As, Bs, method="mixed", tune=False, fallback=True):
    """[x_i] with As[i] x_i = Bs[i] for systems of uneven size, in one launch; also the
    BatchReport. NumPy inputs give NumPy solutions, CUDA tensors give CUDA tensors."""
    if len(As) != len(Bs):
        raise ValueError("solve_batched needs as many right-hand sides as matrices")
    device = bool(As) and _is_torch(As[0]) and As[0].is_cuda
    ns, ks = [], []
    for a, b in zip(As, Bs):
        if a.ndim != 2 or a.shape[0] != a.shape[1]:
            raise ValueError("solve_batched needs square matrices")
        if b.shape[0] != a.shape[0]:
            raise ValueError("a right-hand side's rows must match its matrix")
        ns.append(a.shape[0])
        ks.append(1 if b.ndim == 1 else b.shape[1])
    plan = BatchPlan(ns, ks, method=method, fallback=fallback)
    torch = _torch()
    if device:
        a = torch.cat([x.to(torch.float64).reshape(-1) for x in As]) if As else torch.zeros(0, device="cuda")
        b = torch.cat([x.to(torch.float64).reshape(-1) for x in Bs]) if Bs else torch.zeros(0, device="cuda")
    else:
        a, b = plan.pack([np.asarray(x) for x in As], [np.asarray(x) for x in Bs], device="cuda")
    a, b = a.contiguous(), b.contiguous()
    x = torch.empty(max(plan.b_size, 1), dtype=torch.float64, device=a.device)
    if plan.count:
        if tune:
            plan.tune(a, b, x)
        plan.execute(a, b, x)
    berr, iters, flags, rep = plan.results()
    if rep.no_convergence:
        raise _lib.RmError(_lib.RM_NO_CONVERGENCE, "refinement stalled on some systems and fallback was off")
    xs = plan.unpack(x)
    out = []
    for xi, bi in zip(xs, Bs):
        xi = xi.reshape(bi.shape) if bi.ndim == 1 else xi
        out.append(xi if device else xi.cpu().numpy())
    plan.close()
    return out, rep
