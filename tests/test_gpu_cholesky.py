"""Cholesky on the GPU (rm_dcholesky, rm_dcholesky_batched, rm_dcholesky_solve, linalg.cholesky)
against the oracle's restatement of rustymath's cholesky (core/src/linalg/factor.rs:750-795)
on the reference tests' inputs. Tolerance: each item of L within 8 n eps of the oracle's,
relative to the largest item of its row (the two fold the same products in different
orders); L L^T within 4 eps n of A as tests/linalg.rs:396 asks; exact power-of-two scaling as
tests/linalg.rs:486."""
import ctypes

import numpy as np
import pytest

from oracle import oracle as O
from refdata import distance, norm, ref_random

pytestmark = pytest.mark.gpu
EPS = np.finfo(np.float64).eps


@pytest.fixture(scope="module")
def rb():
    import rustymath_b200 as rb
    return rb


def _spd(n, seed):
    a = ref_random(n, n, seed)
    return O.dgemm(a, a.T) + n * np.eye(n)


def _close_to_oracle(l, lo, n):
    scale = np.abs(lo).max(axis=1, keepdims=True)
    assert (np.abs(l - lo) <= 8 * max(n, 1) * EPS * scale + 1e-300).all()


@pytest.mark.parametrize("n", [1, 2, 5, 31, 32, 33, 63, 64, 65, 71, 130, 530, 1030])
def test_cholesky_matches_the_oracle(rb, n):
    spd = _spd(n, n + 1) if n < 500 else (lambda a: (a + a.T) / 2 + n * np.eye(n))(ref_random(n, n, n))
    l = np.zeros((n, n))
    st = rb._lib.load().rm_dcholesky_host(n, spd.ctypes.data, l.ctypes.data)
    rb._lib.check(st, "cholesky")
    assert (np.triu(l, 1) == 0).all()
    assert distance(O.dgemm(l, l.T), spd, max(norm(spd), 1.0)) < 4 * EPS * max(n, 1)
    _close_to_oracle(l, O.cholesky(spd), n)


@pytest.mark.parametrize("n", [40, 300])
def test_cholesky_scaling_is_exact(rb, n):
    """tests/linalg.rs:485-486 at n = 40 (and a blocked size): scaling A by a power of two c
    (doubled when odd) scales L by sqrt(c) exactly."""
    import torch
    a = ref_random(n, n, 17)
    spd = O.dgemm(a, a.T) + n * np.eye(n)
    tiny = np.finfo(np.float64).tiny / EPS
    quartic = 2.0 ** (int(np.log2(np.finfo(np.float64).max) / 4.0) + 6)
    base = rb.cholesky(torch.tensor(spd, device="cuda"))
    for s in [tiny, 1.0 / tiny, quartic]:
        c = s if np.sqrt(s) * np.sqrt(s) == s else s + s
        got = rb.cholesky(torch.tensor(spd * c, device="cuda"))
        assert torch.equal(got, base * np.sqrt(c))


def test_not_positive_definite(rb):
    from rustymath_b200 import _lib
    n = 70
    neg = -_spd(n, 3)
    l = np.zeros((n, n))
    assert _lib.load().rm_dcholesky_host(n, neg.ctypes.data, l.ctypes.data) == _lib.RM_NOT_POSITIVE_DEFINITE
    # a failure in a later block
    spd = _spd(n, 4)
    spd[66, 66] = -1e6
    assert _lib.load().rm_dcholesky_host(n, spd.ctypes.data, l.ctypes.data) == _lib.RM_NOT_POSITIVE_DEFINITE
    # the Python surface gives NaN, as rustymath's stacks do (tests/test_linalg.py:180-181)
    assert np.isnan(rb.cholesky(-np.eye(2))).all()
    assert np.isnan(rb.cholesky(spd)).all()


def test_stack_one_launch_and_nan_cells(rb):
    """tests/test_linalg.py:229-233: a stack of identities with one cell made indefinite gives
    NaN in that cell only; the rest equal the oracle's factors."""
    from rustymath_b200 import _lib
    a = np.broadcast_to(np.eye(3), (2, 64, 3, 3)).copy()
    a[0, -1, 0, 0] = -1
    l0 = _lib.load().rm_launch_count()
    l = rb.cholesky(a)
    assert _lib.load().rm_launch_count() - l0 == 1
    assert np.isnan(l[0, -1]).all() and np.isfinite(l[1]).all() and np.isfinite(l[0, :-1]).all()
    rng = np.random.default_rng(2)
    stack = np.stack([(lambda m: m @ m.T + 20 * np.eye(20))(rng.standard_normal((20, 20))) for _ in range(50)])
    got = rb.cholesky(stack)
    for i in range(50):
        _close_to_oracle(got[i], O.cholesky(stack[i]), 20)
    assert np.allclose(rb.cholesky(stack[:5].astype(np.float32)), np.linalg.cholesky(stack[:5]), rtol=1e-5)
    assert rb.cholesky(stack.astype(np.float32)).dtype == np.float32


def test_cholesky_solve(rb):
    import torch
    from rustymath_b200 import _lib
    n, k = 400, 5
    spd = _spd(n, 9)
    b = ref_random(n, k, 10)
    ta, tb = torch.tensor(spd, device="cuda"), torch.tensor(b, device="cuda")
    tl = rb.cholesky(ta)
    x = torch.empty_like(tb)
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    _lib.check(_lib.load().rm_dcholesky_solve(n, tl.data_ptr(), tb.data_ptr(), k, x.data_ptr(), s), "solve")
    assert O.backward_error(spd, x.cpu().numpy(), b) <= n * 2.0 ** -53
