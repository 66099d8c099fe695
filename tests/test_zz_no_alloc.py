"""rm_dlu_solve_noalloc: the triangular solves with their scratch in a fixed __device__ array.

It serves callers that cannot allocate device memory during a call (a fixed budget or an
arena that owns all device memory, real-time loops kept away from the allocator). Its
results must equal rm_dlu_solve's, call after call, since both run the same kernels; the
second call checks that leftover scratch from the first does not leak into the result. It
must also allocate nothing: neither the device's stream-ordered pool (where the library's
other entry points take their scratch) nor device memory at large may grow across a call.
This file sorts last so that a failing run has already run every other test."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _solve(lib, name, n, f, p, b, k, trans, x=None):
    import torch
    x = torch.empty_like(b) if x is None else x
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    st = getattr(lib, name)(n, f.data_ptr(), p.data_ptr(), b.data_ptr(), k, x.data_ptr(), trans, s)
    return st, x


def _factors(n, seed):
    import torch
    import rustymath_b200 as rb
    rng = np.random.default_rng(seed)
    a = rng.standard_normal((n, n)) + np.sqrt(n) * np.eye(n)
    fac = rb.lu(torch.tensor(a, device="cuda"))
    return fac.factors.contiguous(), fac.p.contiguous(), rng


@pytest.mark.parametrize("n,k,trans", [(300, 3, 0), (4096, 16, 0), (1000, 5, 1)])
def test_noalloc_matches_rm_dlu_solve(n, k, trans):
    import torch
    from rustymath_b200 import _lib
    lib = _lib.load()
    f, p, rng = _factors(n, n + k)
    for call in range(2):
        b = torch.tensor(rng.standard_normal((n, k)), device="cuda")
        st, want = _solve(lib, "rm_dlu_solve", n, f, p, b, k, trans)
        _lib.check(st, "rm_dlu_solve")
        st, got = _solve(lib, "rm_dlu_solve_noalloc", n, f, p, b, k, trans)
        _lib.check(st, "rm_dlu_solve_noalloc")
        _lib.check(lib.rm_take_status(ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)), "status")
        # the tolerance of the other solve tests: n*eps relative to the solution's scale
        scale = want.abs().max().item()
        assert (got - want).abs().max().item() <= n * np.finfo(np.float64).eps * scale, f"call {call}"


def _default_pool(device):
    from cuda.bindings import driver as cu
    err, pool = cu.cuDeviceGetDefaultMemPool(cu.CUdevice(device))
    assert err == cu.CUresult.CUDA_SUCCESS, err
    return cu, pool


def _pool_attr(cu, pool, attr):
    err, value = cu.cuMemPoolGetAttribute(pool, attr)
    assert err == cu.CUresult.CUDA_SUCCESS, err
    return int(value)


def test_noalloc_allocates_nothing():
    """After a first call (which looks up the array's address and loads the kernels), further
    calls leave the default pool's used bytes where they were, never raise its high-water mark
    above them, and leave the device's free memory unchanged."""
    import torch
    from rustymath_b200 import _lib
    lib = _lib.load()
    n, k = 2048, 8
    f, p, rng = _factors(n, 7)
    b = torch.tensor(rng.standard_normal((n, k)), device="cuda")
    x = torch.empty_like(b)
    st, _ = _solve(lib, "rm_dlu_solve_noalloc", n, f, p, b, k, 0, x)
    _lib.check(st, "rm_dlu_solve_noalloc")
    torch.cuda.synchronize()
    cu, pool = _default_pool(torch.cuda.current_device())
    used = cu.CUmemPool_attribute.CU_MEMPOOL_ATTR_USED_MEM_CURRENT
    high = cu.CUmemPool_attribute.CU_MEMPOOL_ATTR_USED_MEM_HIGH
    used0 = _pool_attr(cu, pool, used)
    # the high-water mark can only be reset to zero; from then on it records the most in use
    err, = cu.cuMemPoolSetAttribute(pool, high, cu.cuuint64_t(0))
    assert err == cu.CUresult.CUDA_SUCCESS, err
    free0 = torch.cuda.mem_get_info()[0]
    for trans in (0, 1, 0):
        st, _ = _solve(lib, "rm_dlu_solve_noalloc", n, f, p, b, k, trans, x)
        _lib.check(st, "rm_dlu_solve_noalloc")
    torch.cuda.synchronize()
    assert _pool_attr(cu, pool, used) == used0
    assert _pool_attr(cu, pool, high) <= used0, "a call took memory from the stream-ordered pool"
    assert torch.cuda.mem_get_info()[0] == free0, "device memory was allocated during a call"


def test_noalloc_reports_a_bad_row_position():
    """A position outside 0..n-1 is skipped by the kernels and reported by rm_take_status."""
    import torch
    from rustymath_b200 import _lib
    lib = _lib.load()
    n, k = 300, 2
    f, p, rng = _factors(n, 11)
    bad = p.clone()
    bad[17] = n + 5
    b = torch.tensor(rng.standard_normal((n, k)), device="cuda")
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert lib.rm_take_status(s) == _lib.RM_OK
    for trans in (0, 1):
        st, _ = _solve(lib, "rm_dlu_solve_noalloc", n, f, bad, b, k, trans)
        assert st == _lib.RM_OK  # asynchronous: the error is found while the kernels run
        assert lib.rm_take_status(s) == _lib.RM_BAD_ARG
        assert lib.rm_take_status(s) == _lib.RM_OK  # read once, then cleared
    st, got = _solve(lib, "rm_dlu_solve_noalloc", n, f, p, b, k, 0)
    _lib.check(st, "rm_dlu_solve_noalloc")
    assert lib.rm_take_status(s) == _lib.RM_OK
    want = torch.linalg.solve(torch.tensor(_lu_matrix(f, p)), b.cpu())
    assert (got.cpu() - want).abs().max().item() <= 1e-10 * want.abs().max().item()


def _lu_matrix(f, p):
    """The matrix P^T L U that column-major factors and row positions describe."""
    fa = f.cpu().numpy().T
    n = fa.shape[0]
    lu = np.tril(fa, -1) + np.eye(n), np.triu(fa)
    a = np.empty((n, n))
    a[p.cpu().numpy()] = lu[0] @ lu[1]
    return a


def test_noalloc_rejects_sizes_beyond_its_scratch():
    from rustymath_b200 import _lib
    lib = _lib.load()
    big = 4097
    assert lib.rm_dlu_solve_noalloc(big, None, None, None, 1, None, 0, None) == _lib.RM_BAD_ARG
    assert lib.rm_dlu_solve_noalloc(10, None, None, None, 17, None, 0, None) == _lib.RM_BAD_ARG
