"""rm_dlu_solve_noalloc: the triangular solves with their scratch in a fixed __device__ array.

It serves callers that cannot allocate device memory during a call (a fixed budget or an
arena that owns all device memory, real-time loops kept away from the allocator). Its
results must equal rm_dlu_solve's, call after call, since both run the same kernels; the
second call checks that leftover scratch from the first does not leak into the result.
This file sorts last so that a failing run has already run every other test."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _solve(lib, name, n, f, p, b, k, trans):
    import torch
    x = torch.empty_like(b)
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    st = getattr(lib, name)(n, f.data_ptr(), p.data_ptr(), b.data_ptr(), k, x.data_ptr(), trans, s)
    return st, x


@pytest.mark.parametrize("n,k,trans", [(300, 3, 0), (4096, 16, 0), (1000, 5, 1)])
def test_noalloc_matches_rm_dlu_solve(n, k, trans):
    import torch
    import rustymath_b200 as rb
    from rustymath_b200 import _lib
    lib = _lib.load()
    rng = np.random.default_rng(n + k)
    a = rng.standard_normal((n, n)) + np.sqrt(n) * np.eye(n)
    fac = rb.lu(torch.tensor(a, device="cuda"))
    f, p = fac.factors.contiguous(), fac.p.contiguous()
    for call in range(2):
        b = torch.tensor(rng.standard_normal((n, k)), device="cuda")
        st, want = _solve(lib, "rm_dlu_solve", n, f, p, b, k, trans)
        _lib.check(st, "rm_dlu_solve")
        st, got = _solve(lib, "rm_dlu_solve_noalloc", n, f, p, b, k, trans)
        _lib.check(st, "rm_dlu_solve_noalloc")
        torch.cuda.synchronize()
        # the tolerance of the other solve tests: n*eps relative to the solution's scale
        scale = want.abs().max().item()
        assert (got - want).abs().max().item() <= n * np.finfo(np.float64).eps * scale, f"call {call}"


def test_noalloc_rejects_sizes_beyond_its_scratch():
    from rustymath_b200 import _lib
    lib = _lib.load()
    big = 4097
    assert lib.rm_dlu_solve_noalloc(big, None, None, None, 1, None, 0, None) == _lib.RM_BAD_ARG
    assert lib.rm_dlu_solve_noalloc(10, None, None, None, 17, None, 0, None) == _lib.RM_BAD_ARG
