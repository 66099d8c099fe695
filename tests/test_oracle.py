"""The CPU oracle against the reference's own known answers and property tests.

Each test restates a check from rustymath's tests/linalg.rs or tests/test_linalg.py (cited
per test) on the same inputs (tests/refdata.py regenerates the reference's test matrices),
so the oracle's parity with the reference is pinned before it checks the GPU path."""
import json
import os

import numpy as np
import pytest
import scipy.linalg as sl

from oracle import oracle as O
from refdata import distance, lower_of, norm, ref_random, upper_of

EPS = np.finfo(np.float64).eps
KC, MC, NC = 256, 128, 2048
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def product(a, b):
    return O.dgemm(a, b)


@pytest.mark.parametrize("size", [[0, 3, 4], [3, 0, 4], [3, 4, 0], [1, 1, 1], [5, 7, 9],
                                  [MC + 3, KC + 5, 37], [MC + 3, KC + 5, 1], [17, 3, NC + 5]])
def test_products_match_folds_in_order(size):
    """tests/linalg.rs:160-205: exact equality with an in-order fold on small integers."""
    m, k, n = size
    a = np.array([(i * 7 % 17) - 8.0 for i in range(m * k)]).reshape(m, k)
    b = np.array([(i * 5 % 13) - 6.0 for i in range(k * n)]).reshape(k, n)
    expected = a.astype(np.int64) @ b.astype(np.int64)
    into = np.ones((m, n))
    got = O.dgemm(a, b, c=into, beta=0.0)
    assert np.array_equal(got, expected.astype(np.float64))
    assert np.array_equal(O.dgemm_fold(a, b), expected.astype(np.float64))


def test_packed_product_is_the_in_order_fold():
    """The packed product folds each item in k order (core/src/linalg.rs:1419-1441), so its
    bits equal the plain fold's at any blocking and thread count."""
    rng = np.random.default_rng(3)
    a, b, c = rng.standard_normal((70, 300)), rng.standard_normal((300, 45)), rng.standard_normal((70, 45))
    for threads in [1, 4]:
        O.set_threads(threads)
        assert np.array_equal(O.dgemm(a, b, alpha=-1.0, beta=1.0, c=c), O.dgemm_fold(a, b, -1.0, 1.0, c))
    O.set_threads(0)


@pytest.mark.parametrize("n", [0, 1, 2, 5, 31, 32, 33, 71])
def test_decompositions(n):
    """tests/linalg.rs:373-390: LU, solve and inverse residuals below 4*eps*n."""
    bound = 4 * EPS * max(n, 1)
    a = ref_random(n, n, n + 1)
    f, p = O.lu_factor(a)
    l, u = lower_of(f), upper_of(f)
    pa = a[p] if n else a
    assert distance(product(l, u), pa, max(norm(a), 1.0)) < bound
    for k in [1, 3]:
        b = ref_random(n, k, 99)
        x = O.lu_solve(f, p, b)
        assert distance(product(a, x), b, max(norm(a) * norm(x), 1.0)) < bound
    inv = O.lu_inverse(f, p)
    assert distance(product(a, inv), np.eye(n), max(norm(a) * norm(inv), 1.0)) < bound


def test_hard_matrices_scaling():
    """tests/linalg.rs:466-483: scaling by a power of two scales the factors exactly."""
    n = 40
    tiny = np.finfo(np.float64).tiny / EPS
    quartic = 2.0 ** (int(np.log2(np.finfo(np.float64).max) / 4.0) + 6)
    a, b = ref_random(n, n, 17), ref_random(n, 3, 19)
    f, fp = O.lu_factor(a)
    for s in [tiny, 1.0 / tiny, quartic]:
        g, gp = O.lu_factor(a * s)
        assert np.array_equal(gp, fp)
        i, j = np.indices((n, n))  # factors[j][i] holds item (i, j); upper where i <= j
        want = np.where(j <= i, f * s, f)
        assert np.array_equal(g, want)
        assert np.array_equal(O.lu_solve(g, gp, b * s), O.lu_solve(f, fp, b))
        assert np.array_equal(O.lu_inverse(g, gp) * s, O.lu_inverse(f, fp))


@pytest.mark.parametrize("zero", [0, 35, 70])
def test_zero_column(zero):
    """tests/linalg.rs:501-508: a zero column gives finite factors with a zero pivot."""
    n = 71
    a = ref_random(n, n, 29)
    a[:, zero] = 0.0
    f, p = O.lu_factor(a)
    assert np.isfinite(f).all() and (np.diag(f) == 0.0).any()
    assert distance(product(lower_of(f), upper_of(f)), a[p], norm(a)) < 4 * EPS * n


def test_subnormal_pivot():
    """tests/linalg.rs:510-511: lu([p, 1, q, 1]) = [p, q/p, 1, 1 - q/p] for subnormal p, q."""
    tiny = np.finfo(np.float64).tiny
    p, q = tiny / 1024.0, tiny / 1048576.0
    f, _ = O.lu_factor(np.array([[p, 1.0], [q, 1.0]]))
    assert f.reshape(-1).tolist() == [p, q / p, 1.0, 1.0 - q / p]


def test_determinants():
    """tests/linalg.rs:548-558: known determinants and the singular inverse."""
    swapped = np.array([0., 2, 0, 0, 1, 0, 0, 0, 0, 0, 3, 0, 0, 0, 0, 4]).reshape(4, 4)
    f, p = O.lu_factor(swapped)
    assert O.lu_determinant(f, p) == -24.0
    singular = np.array([[1.0, 0.0], [3.0, 0.0]])
    f, p = O.lu_factor(singular)
    assert O.lu_determinant(f, p) == 0.0
    assert O.lu_log_determinant(f, p) == (0.0, -np.inf)
    bad = np.array([[1.0, 2.0], [2.0, 4.0]])
    f, _ = O.lu_factor(bad)
    assert not O.regular(bad, f)
    assert O.solve(bad, np.ones(2)) is None
    regular = ref_random(6, 6, 11)
    f, p = O.lu_factor(regular)
    sign, log = O.lu_log_determinant(f, p)
    assert abs(sign * np.exp(log) / O.lu_determinant(f, p) - 1.0) < 64 * 4 * EPS


@pytest.mark.parametrize("n", [530, 1030])
def test_blocked(n):
    """tests/linalg.rs:569-583: O(n^2) residual checks through random vectors."""
    bound = 4 * EPS * n
    a = ref_random(n, n, n)
    x = ref_random(n, 1, 3)
    f, p = O.lu_factor(a)
    l, u = lower_of(f), upper_of(f)
    ax = product(a, x)
    assert distance(product(l, product(u, x)), ax[p], norm(a) * norm(x)) < bound
    b = ref_random(n, 3, 5)
    solved = O.lu_solve(f, p, b)
    assert distance(product(a, solved), b, norm(a) * norm(solved)) < bound
    inv = O.lu_inverse(f, p)
    assert distance(product(a, product(inv, x)), x, norm(a) * norm(inv) * norm(x)) < bound


def test_python_lu_base_stack():
    """tests/test_linalg.py:6-32 at float64: the base matrix stack against NumPy."""
    base = np.array([[0., 2, 1], [3, 1, -1], [1, 0, 4]])
    b = np.arange(12.).reshape(3, 4)[:, ::-1]
    for k in range(64):
        a = base + k / 8 * np.eye(3)
        f, p = O.lu_factor(a)
        assert np.allclose(lower_of(f) @ upper_of(f), a[p], rtol=0.002, atol=0.002)
        assert np.allclose(O.lu_solve(f, p, b), np.linalg.solve(a, b), rtol=0.003, atol=0.003)
        assert np.allclose(O.lu_inverse(f, p), np.linalg.inv(a), rtol=0.003, atol=0.003)
        assert np.allclose(O.lu_determinant(f, p), np.linalg.det(a), rtol=0.003, atol=0.003)
        sign, log = O.lu_log_determinant(f, p)
        want = np.linalg.slogdet(a)
        assert np.allclose(sign, want.sign) and np.allclose(log, want.logabsdet)


def test_linalg_vs_numpy():
    """tests/test_linalg.py:94-104 at float64: default_rng(0) stacks against NumPy."""
    rng = np.random.default_rng(0)
    a, b = rng.standard_normal((4, 5, 5)), rng.standard_normal((4, 5, 3))
    for i in range(4):
        assert np.allclose(O.solve(a[i], b[i]), np.linalg.solve(a[i], b[i]))
        assert np.allclose(O.dgemm(a[i], b[i]), a[i] @ b[i])


@pytest.mark.parametrize("n", [3, 17, 64, 100, 257])
def test_pivots_match_lapack(n):
    """Partial pivoting picks the same rows as LAPACK getrf (an independent statement of
    the same rule) on matrices without near ties."""
    a = np.random.default_rng(n).standard_normal((n, n))
    f, piv = O.lu_pivots(a)
    lu, lpiv = sl.lu_factor(a)
    assert np.array_equal(piv, lpiv)
    assert np.allclose(f.T, lu, rtol=1e-10, atol=1e-12)


def test_solve_transposed():
    n = 37
    a = ref_random(n, n, 5)
    b = ref_random(n, 2, 6)
    f, p = O.lu_factor(a)
    x = O.lu_solve_transposed(f, p, b)
    assert np.allclose(a.T @ x, b, rtol=1e-12, atol=1e-12)


def test_backward_error_of_exact_solution_is_zero():
    a = np.array([[2.0, 1.0], [1.0, 3.0]])
    x = np.array([1.0, 2.0])
    assert O.backward_error(a, x, a @ x) == 0.0
    assert O.backward_error(a, x + 1e-3, a @ x) > 1e-5


def test_golden_fixtures():
    """The committed known-answer fixtures (tests/golden/make_golden.py) hold for the oracle."""
    with open(os.path.join(GOLDEN, "known_answers.json")) as fh:
        cases = json.load(fh)
    for case in cases:
        a = np.array(case["a"], dtype=np.float64)
        f, p = O.lu_factor(a)
        if "factors" in case:
            assert f.reshape(-1).tolist() == case["factors"], case["name"]
        if "perm" in case:
            assert p.tolist() == case["perm"], case["name"]
        if "det" in case:
            assert O.lu_determinant(f, p) == case["det"], case["name"]
        if "regular" in case:
            assert O.regular(a, f) == case["regular"], case["name"]


def _spd(n, seed):
    """tests/linalg.rs:391-392: A A^T + n I from the reference's random matrix."""
    a = ref_random(n, n, seed)
    return product(a, a.T) + n * np.eye(n)


@pytest.mark.parametrize("n", [0, 1, 2, 5, 31, 32, 33, 71])
def test_cholesky_decompositions(n):
    """tests/linalg.rs:391-399: L is lower triangular, L L^T within 4 eps n of the matrix, and
    a negative definite matrix has no factor."""
    spd = _spd(n, n + 1)
    l = O.cholesky(spd)
    assert l is not None
    assert (np.triu(l, 1) == 0).all()
    assert distance(product(l, l.T), spd, max(norm(spd), 1.0)) < 4 * EPS * max(n, 1)
    if n > 0:
        assert O.cholesky(-spd) is None


@pytest.mark.parametrize("n", [530, 1030])
def test_cholesky_blocked(n):
    """tests/linalg.rs:584-589: (A + A^T)/2 + n I through random vectors."""
    a = ref_random(n, n, n)
    x = ref_random(n, 1, 3)
    spd = (a + a.T) / 2 + n * np.eye(n)
    l = O.cholesky(spd)
    assert (np.triu(l, 1) == 0).all()
    assert distance(product(l, product(l.T, x)), product(spd, x), norm(spd) * norm(x)) < 4 * EPS * n


def test_cholesky_scaling_is_exact():
    """tests/linalg.rs:485-486: a power-of-two scale c (doubled when odd) scales L by sqrt(c)
    exactly."""
    n = 40
    a = ref_random(n, n, 17)
    spd = product(a, a.T) + n * np.eye(n)
    tiny = np.finfo(np.float64).tiny / EPS
    quartic = 2.0 ** (int(np.log2(np.finfo(np.float64).max) / 4.0) + 6)
    base = O.cholesky(spd)
    for s in [tiny, 1.0 / tiny, quartic]:
        c = s if np.sqrt(s) * np.sqrt(s) == s else s + s
        assert np.array_equal(O.cholesky(spd * c), base * np.sqrt(c))


def test_cholesky_vs_numpy():
    """tests/test_linalg.py:109-110: a a^T + 5 I against numpy.linalg.cholesky."""
    a = np.random.default_rng(0).standard_normal((5, 5))
    spd = a @ a.T + 5 * np.eye(5)
    assert np.allclose(O.cholesky(spd), np.linalg.cholesky(spd))
    assert O.cholesky(-np.eye(2)) is None
