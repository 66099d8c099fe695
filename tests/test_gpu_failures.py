"""Failure detection without a GPU fault.

- A bounded device-side wait that runs out: rm_test_chain_timeout runs a small chain solve
  whose first block never runs, with a 1 ms wait limit passed to the kernel; the kernel gives
  up, reports RM_TIMEOUT through a status word and returns, and the device keeps working.
- Host-side failures of the allocator (out of memory, a CUDA error) made by
  rm_test_inject_failure: each entry point returns the matching status, frees what it holds,
  and the next call succeeds.
- A row position outside 0..n-1 handed to the asynchronous rm_dlu_solve: the kernels skip it
  and rm_take_status reports it.
Nothing here faults, traps or hangs a GPU."""
import ctypes
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _lib():
    from rustymath_b200 import _lib
    return _lib, _lib.load()


def _solve_ok(n=200, k=2, method="plain"):
    import rustymath_b200 as rb
    rng = np.random.default_rng(n)
    a = rng.standard_normal((n, n)) + n * np.eye(n)
    b = rng.standard_normal((n, k))
    x = rb.solve(a, b, method=method)
    assert np.abs(a @ x - b).max() <= 1e-10 * np.abs(b).max()


def test_a_wait_that_runs_out_reports_timeout_and_the_device_survives():
    _l, lib = _lib()
    t0 = time.perf_counter()
    st = lib.rm_test_chain_timeout(1_000_000)  # 1 ms
    dt = time.perf_counter() - t0
    assert st == _l.RM_TIMEOUT, _l.last_error()
    assert dt < 1.0, f"the expired waits took {dt:.3f} s"
    _solve_ok()
    assert lib.rm_test_chain_timeout(50_000) == _l.RM_TIMEOUT
    _solve_ok(method="mixed")


@pytest.mark.parametrize("kind,status", [("RM_INJECT_OUT_OF_MEMORY", "RM_OUT_OF_MEMORY"),
                                         ("RM_INJECT_CUDA_ERROR", "RM_CUDA_ERROR")])
def test_allocation_failures_are_reported(kind, status):
    import rustymath_b200 as rb
    _l, lib = _lib()
    n, k = 150, 3
    rng = np.random.default_rng(3)
    a = rng.standard_normal((n, n)) + n * np.eye(n)
    b = rng.standard_normal((n, k))
    x = np.zeros((n, k))
    opts = rb.linalg._options("plain")
    rep = _l.SolveReport()
    assert lib.rm_test_inject_failure(getattr(_l, kind), 0, 1) == _l.RM_OK
    st = lib.rm_dsolve_host(n, a.ctypes.data, b.ctypes.data, k, x.ctypes.data, ctypes.byref(opts), ctypes.byref(rep))
    assert st == getattr(_l, status)
    # the Python surface raises for it
    assert lib.rm_test_inject_failure(getattr(_l, kind), 0, 1) == _l.RM_OK
    with pytest.raises(_l.RmError) as e:
        rb.solve(a, b)
    assert e.value.status == getattr(_l, status)
    # armed for one event only: the next call works
    _solve_ok(n, k)
    # a failure deeper in a call: the host-pointer solve's own buffers are allocated, the plain
    # solve's scratch inside it is not; the call returns the status and frees its buffers
    assert lib.rm_test_inject_failure(getattr(_l, kind), 1, 1) == _l.RM_OK
    st = lib.rm_dsolve_host(n, a.ctypes.data, b.ctypes.data, k, x.ctypes.data, ctypes.byref(opts), ctypes.byref(rep))
    assert st == getattr(_l, status)
    # the same inside the mixed solve
    mixed = rb.linalg._options("mixed")
    assert lib.rm_test_inject_failure(getattr(_l, kind), 1, 1) == _l.RM_OK
    st = lib.rm_dsolve_host(n, a.ctypes.data, b.ctypes.data, k, x.ctypes.data, ctypes.byref(mixed), ctypes.byref(rep))
    assert st == getattr(_l, status)
    # disarmed, both methods work again
    assert lib.rm_test_inject_failure(getattr(_l, kind), 0, 0) == _l.RM_OK
    _solve_ok(n, k)
    _solve_ok(n, k, method="mixed")


@pytest.mark.parametrize("n", [100, 257])
def test_a_bad_row_position_is_reported_by_take_status(n):
    """n = 100 takes the one-CTA solve without a transpose, n = 257 the block-chained solves."""
    import torch
    import rustymath_b200 as rb
    _l, lib = _lib()
    k = 3
    rng = np.random.default_rng(5)
    a = torch.tensor(rng.standard_normal((n, n)) + n * np.eye(n), device="cuda")
    fac = rb.lu(a)
    bad = fac.p.clone()
    bad[n // 2] = -1
    b = torch.tensor(rng.standard_normal((n, k)), device="cuda")
    x = torch.empty_like(b)
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert lib.rm_take_status(s) == _l.RM_OK
    for trans in (0, 1):
        st = lib.rm_dlu_solve(n, fac.factors.data_ptr(), bad.data_ptr(), b.data_ptr(), k, x.data_ptr(), trans, s)
        assert st == _l.RM_OK
        assert lib.rm_take_status(s) == _l.RM_BAD_ARG
    assert lib.rm_take_status(s) == _l.RM_OK
    # the Python surface checks positions before it calls
    with pytest.raises(IndexError):
        rb.lu_solve(fac.factors, bad, b)
    x = rb.lu_solve(fac.factors, fac.p, b)
    assert (a @ x - b).abs().max().item() <= 1e-10 * b.abs().max().item()
