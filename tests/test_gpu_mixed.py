"""The mixed-precision solve (RM_METHOD_F32_IR): float32 LU on the tensor cores with panels
pivoted among their own 256 rows, then float64 refinement. Its results must meet the plain path's bar: normwise
backward error <= n * 2^-53, measured here by the oracle's double-double residual, and a
solution that agrees with the oracle's within the forward error kappa * n * eps allows."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu
EPS = np.finfo(np.float64).eps


def conditioned(n, k, kappa, seed):
    """A = U diag(logspace(0, -log10 kappa)) V^T with Haar-like U, V; B ~ N(0,1)."""
    rng = np.random.default_rng(seed)
    u, _ = np.linalg.qr(rng.standard_normal((n, n)))
    v, _ = np.linalg.qr(rng.standard_normal((n, n)))
    s = np.logspace(0, -np.log10(kappa), n)
    return (u * s) @ v.T, rng.standard_normal((n, k))


@pytest.fixture(scope="module")
def rb():
    import rustymath_b200 as rb
    return rb


@pytest.mark.parametrize("n,k,kappa", [(1024, 16, 1e4), (1001, 3, 1e4), (130, 1, 1e3), (17, 2, 10.0), (5, 1, 2.0),
                                       (2048, 5, 1e4), (1500, 17, 1e3), (1100, 17, 1e3), (1536, 16, 1e4),
                                       (1200, 8, 1e3)])
def test_mixed_meets_the_fp64_bar(rb, n, k, kappa):
    a, b = conditioned(n, k, kappa, n + k)
    x, reps = rb.solve_report(a, b, method="mixed")
    rep = reps[0]
    assert rep.method_used == 1 and rep.fell_back == 0, "classical refinement converged"
    assert rep.iterations <= 5
    assert O.backward_error(a, x, b) <= n * 2.0 ** -53
    xo = O.solve(a, b)
    assert np.abs(x - xo).max() / np.abs(xo).max() <= kappa * n * EPS


def test_mixed_device_tensors(rb):
    import torch
    n, k = 600, 4
    a, b = conditioned(n, k, 1e3, 3)
    x = rb.solve(torch.tensor(a, device="cuda"), torch.tensor(b, device="cuda"), method="mixed")
    assert O.backward_error(a, x.cpu().numpy(), b) <= n * 2.0 ** -53


def test_mixed_beyond_float32_reach(rb):
    """kappa = 1e12 is beyond float32 factors' reach (kappa * u >> 1): classical refinement
    stalls; GMRES-IR or, failing it, the plain float64 LU answers, as the report says."""
    n, k = 300, 2
    a, b = conditioned(n, k, 1e12, 5)
    x, reps = rb.solve_report(a, b, method="mixed")
    assert reps[0].method_used in (0, 2)
    assert reps[0].fell_back == (1 if reps[0].method_used == 0 else 0)
    assert O.backward_error(a, x, b) <= n * 2.0 ** -53


@pytest.mark.parametrize("kappa,restart", [(3e7, 20), (1e8, 60)])
def test_gmres_ir_where_classical_refinement_stalls(rb, kappa, restart):
    """kappa * u_f near or above 1: classical refinement with float32 factors stalls, while
    flexible GMRES right-preconditioned by the same factors converges (GMRES-IR); at 1e8 it
    needs a longer restart cycle."""
    import ctypes
    from rustymath_b200 import _lib
    n, k = 401, 3  # odd n: the float64 products take a padded copy of A
    a, b = conditioned(n, k, kappa, 11)
    lib = _lib.load()
    x = np.zeros((n, k))
    opts = rb.linalg._options("mixed", gmres_restart=restart)
    rep = _lib.SolveReport()
    st = lib.rm_dsolve_host(n, a.ctypes.data, b.ctypes.data, k, x.ctypes.data, ctypes.byref(opts), ctypes.byref(rep))
    assert st == 0 and rep.method_used == _lib.RM_METHOD_GMRES_IR and rep.fell_back == 0
    assert O.backward_error(a, x, b) <= n * 2.0 ** -53
    # with GMRES-IR switched off, the float64 fallback answers instead
    x2 = np.zeros((n, k))
    opts = rb.linalg._options("mixed", gmres_restart=0)
    st = lib.rm_dsolve_host(n, a.ctypes.data, b.ctypes.data, k, x2.ctypes.data, ctypes.byref(opts),
                            ctypes.byref(rep))
    assert st == 0 and rep.fell_back == 1 and rep.method_used == 0
    assert O.backward_error(a, x2, b) <= n * 2.0 ** -53


def test_mixed_singular_matrix_is_not_regular(rb):
    """A singular matrix: refinement fails, the fallback applies rustymath's regular test."""
    a = np.ones((8, 8))
    with pytest.raises(rb.NotRegular):
        rb.solve(a, np.ones(8), method="mixed")


def test_mixed_without_fallback_reports_no_convergence(rb):
    import ctypes
    from rustymath_b200 import _lib
    n, k = 200, 1
    a, b = conditioned(n, k, 1e12, 7)
    x = np.zeros((n, k))
    opts = rb.linalg._options("mixed", fallback=False)
    rep = _lib.SolveReport()
    st = _lib.load().rm_dsolve_host(n, a.ctypes.data, b.ctypes.data, k, x.ctypes.data, ctypes.byref(opts),
                                    ctypes.byref(rep))
    assert st == _lib.RM_NO_CONVERGENCE


def test_window_without_a_good_pivot(rb):
    """The mixed factorization pivots each 128-column panel among its own 256 rows. With the
    first 256 rows scaled by 1e-8 the first panels find only tiny candidates in their window,
    while the large entries sit below it: the float32 factors grow and classical refinement
    cannot recover. The solve must still meet the float64 bar through one of its other routes
    (GMRES-IR, or the plain float64 LU after fallback), and the report must say which."""
    n, k = 1024, 3
    a, b = conditioned(n, k, 1e2, 11)
    a[:256] *= 1e-8
    x, reps = rb.solve_report(a, b, method="mixed")
    rep = reps[0]
    assert rep.method_used in (0, 1, 2)
    assert rep.fell_back == (1 if rep.method_used == 0 else 0)
    assert O.backward_error(a, x, b) <= n * 2.0 ** -53
    print(f"window test: method_used={rep.method_used} iterations={rep.iterations} fell_back={rep.fell_back}")
