"""rm_dtrsm, the triangular solve behind the reference's xtrsm seam, against SciPy's
solve_triangular (LAPACK) on every side/uplo/trans/diag combination: agreement within the
forward error cond(op(A)) * n * eps allows."""
import ctypes
import itertools

import numpy as np
import pytest
from scipy.linalg import solve_triangular

pytestmark = pytest.mark.gpu
EPS = np.finfo(np.float64).eps


@pytest.mark.parametrize("side,uplo,trans,diag", list(itertools.product((141, 142), (121, 122), (111, 112),
                                                                         (131, 132))))
@pytest.mark.parametrize("m,n", [(70, 33), (200, 17), (1, 5), (129, 1)])
def test_trsm_matches_lapack(side, uplo, trans, diag, m, n):
    import torch
    from rustymath_b200 import _lib
    rng = np.random.default_rng(m * n + side + uplo + trans + diag)
    order = m if side == 141 else n
    a = rng.standard_normal((order, order)) / np.sqrt(order) + 2 * np.eye(order)
    a[np.triu_indices(order, 1) if uplo == 122 else np.tril_indices(order, -1)] = np.nan  # never read
    x = rng.standard_normal((m, n))
    tri = np.tril(np.nan_to_num(a)) if uplo == 122 else np.triu(np.nan_to_num(a))
    if diag == 132:
        np.fill_diagonal(tri, 1.0)
    op = tri.T if trans == 112 else tri
    want = np.linalg.solve(op, x) if side == 141 else np.linalg.solve(op.T, x.T).T
    ta = torch.tensor(a, device="cuda")
    tx = torch.tensor(x, device="cuda")
    st = _lib.load().rm_dtrsm(side, uplo, trans, diag, m, n, ta.data_ptr(), order, tx.data_ptr(), n,
                              ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    _lib.check(st, "rm_dtrsm")
    got = tx.cpu().numpy()
    assert np.abs(got - want).max() <= np.linalg.cond(op) * order * 8 * EPS * max(np.abs(want).max(), 1.0)
    if side == 141:
        ref = solve_triangular(tri, x, lower=uplo == 122, trans=1 if trans == 112 else 0, unit_diagonal=diag == 132)
        assert np.allclose(got, ref, rtol=1e-10, atol=1e-12)


def test_trsm_bad_codes():
    from rustymath_b200 import _lib
    assert _lib.load().rm_dtrsm(140, 121, 111, 131, 2, 2, None, 2, None, 2, None) == _lib.RM_BAD_ARG


def test_trsm_host_form():
    from rustymath_b200 import _lib
    rng = np.random.default_rng(9)
    m, n = 90, 7
    a = np.tril(rng.standard_normal((n, n))) + 3 * np.eye(n)
    x = rng.standard_normal((m, n))
    want = np.linalg.solve(a.T, x.T).T  # x a^-1: side right, lower, no transpose, non-unit
    got = x.copy()
    st = _lib.load().rm_dtrsm_host(142, 122, 111, 131, m, n, a.ctypes.data, n, got.ctypes.data, n)
    _lib.check(st, "rm_dtrsm_host")
    assert np.allclose(got, want, rtol=1e-12, atol=1e-12)
