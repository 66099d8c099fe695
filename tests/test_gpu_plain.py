"""Parity of the plain float64 GPU path (C ABI through rustymath_b200) with the oracle.

Each case compares the CUDA result with the CPU oracle (a restatement of rustymath's
algorithms) on the same seeded inputs, or checks a known answer from rustymath's own
tests (cited). Tolerances are stated per test: exact for integer-valued products and for
power-of-two scaling; n*eps relative for the well-conditioned solve; 4*eps*n residuals as
in tests/linalg.rs elsewhere."""
import numpy as np
import pytest

from oracle import oracle as O
from refdata import distance, lower_of, norm, ref_random, upper_of

pytestmark = pytest.mark.gpu

EPS = np.finfo(np.float64).eps
KC, MC, NC = 256, 128, 2048


@pytest.fixture(scope="module")
def rb():
    import rustymath_b200 as rb
    rb._lib.load()
    return rb


def product(a, b):
    return O.dgemm(a, b)


# ---------------------------------------------------------------- GEMM

@pytest.mark.parametrize("size", [[0, 3, 4], [3, 0, 4], [3, 4, 0], [1, 1, 1], [5, 7, 9], [MC + 3, KC + 5, 37],
                                  [MC + 3, KC + 5, 1], [17, 3, NC + 5], [129, 33, 257], [300, 17, 130]])
def test_gemm_exact_integers(rb, size):
    """tests/linalg.rs:160-205: small whole numbers make every sum exact in any order."""
    m, k, n = size
    a = np.array([(i * 7 % 17) - 8.0 for i in range(m * k)]).reshape(m, k)
    b = np.array([(i * 5 % 13) - 6.0 for i in range(k * n)]).reshape(k, n)
    expected = (a.astype(np.int64) @ b.astype(np.int64)).astype(np.float64)
    assert np.array_equal(rb.matmul(a, b), expected)


@pytest.mark.parametrize("ta,tb", [(0, 0), (0, 1), (1, 0), (1, 1)])
@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (7, 9, 5), (64, 64, 64), (100, 130, 70), (257, 129, 300),
                                   (512, 512, 512), (1000, 700, 33)])
def test_gemm_random(rb, ta, tb, m, n, k):
    """alpha op(A) op(B) + beta C against the oracle; |error| <= 2k eps |A||B| elementwise."""
    import ctypes
    rng = np.random.default_rng(m * 1000 + n * 10 + k)
    a = rng.uniform(-1, 1, (k, m) if ta else (m, k))
    b = rng.uniform(-1, 1, (n, k) if tb else (k, n))
    c = rng.uniform(-1, 1, (m, n))
    alpha, beta = -1.5, 0.5
    got = c.copy()
    lib = rb._lib.load()
    st = lib.rm_dgemm_host(ta, tb, m, n, k, alpha, a.ctypes.data, a.shape[1], b.ctypes.data, b.shape[1], beta,
                           got.ctypes.data, n)
    rb._lib.check(st, "dgemm")
    want = O.dgemm(a, b, alpha=alpha, beta=beta, c=c, ta=bool(ta), tb=bool(tb))
    bound = 2 * k * EPS * (np.abs(alpha) * (np.abs(a.T if ta else a) @ np.abs(b.T if tb else b)) + abs(beta) * np.abs(c))
    assert (np.abs(got - want) <= bound + 1e-300).all()


def test_gemm_unaligned_leading_dimensions(rb):
    """Odd leading dimensions take the copying route; the result is unchanged."""
    rng = np.random.default_rng(5)
    big_a, big_b = rng.standard_normal((40, 37)), rng.standard_normal((37, 41))
    a, b = big_a[:, :33], big_b[:33, :29]
    got = np.zeros((40, 29))
    lib = rb._lib.load()
    st = lib.rm_dgemm_host(0, 0, 40, 29, 33, 1.0, big_a.ctypes.data, 37, big_b.ctypes.data, 41, 0.0, got.ctypes.data, 29)
    rb._lib.check(st, "dgemm")
    assert np.allclose(got, a @ b, rtol=1e-13, atol=1e-13)


def test_gemm_bad_arguments(rb):
    lib = rb._lib.load()
    assert lib.rm_dgemm_host(0, 0, -1, 2, 2, 1.0, None, 2, None, 2, 0.0, None, 2) == rb._lib.RM_BAD_ARG
    assert lib.rm_dgemm_host(0, 0, 2, 2, 2, 1.0, None, 1, None, 2, 0.0, None, 2) == rb._lib.RM_BAD_ARG


# ---------------------------------------------------------------- LU

@pytest.mark.parametrize("n", [1, 2, 5, 31, 32, 33, 71, 127, 128, 129, 200, 257, 530, 1030])
def test_lu_matches_oracle(rb, n):
    """Pivots equal the oracle's; factors agree to 64*n*eps of their scale; the residual
    ||LU - PA|| stays below the reference's 4*eps*n (tests/linalg.rs:373-382)."""
    a = ref_random(n, n, n + 1)
    f, p = rb.lu(a)
    fo, po = O.lu_factor(a)
    assert np.array_equal(p, po)
    assert np.abs(f - fo).max() <= 64 * n * EPS * max(1.0, np.abs(fo).max())
    assert distance(product(lower_of(f), upper_of(f)), a[p], max(norm(a), 1.0)) < 4 * EPS * max(n, 1)


@pytest.mark.parametrize("n", [1, 2, 5, 31, 32, 33, 64, 71, 100, 128, 129, 200, 255, 256])
def test_small_lu_is_the_oracles_bits(rb, n):
    """Up to n = 256 the factorization is one cluster launch in which every item takes one fma
    per pivot column in column order, which is how rustymath's lu_factor reaches it through
    its packed products' in-order folds (core/src/linalg/factor.rs:580-630,
    core/src/linalg.rs:1282): factors and positions are the oracle's, bit for bit, on the
    reference tests' inputs and on N(0,1) matrices."""
    for a in (ref_random(n, n, n + 1), np.random.default_rng(n).standard_normal((n, n))):
        f, p = rb.lu(a)
        fo, po = O.lu_factor(a)
        assert np.array_equal(p, po)
        assert np.array_equal(f, fo)


@pytest.mark.parametrize("n", [1, 2, 5, 32, 33, 71, 100, 128, 191, 192])
def test_small_solve_is_the_oracles_bits(rb, n):
    """Up to n = 192 with one right-hand side, solve is the oracle's LuWork::solve bit for bit:
    the factors as above, then the single-column triangular solves in rustymath's order
    (core/src/linalg/factor.rs:725-748). With 2..8 right-hand sides each column is solved the
    same way, within n*eps of the oracle (which takes its blocked route there)."""
    rng = np.random.default_rng(40 + n)
    for a in (ref_random(n, n, n + 1), rng.standard_normal((n, n)) + n * np.eye(n)):
        b = rng.standard_normal((n, 1))
        assert np.array_equal(rb.solve(a, b), O.solve(a, b))
        b3 = rng.standard_normal((n, 3))
        x3, xo3 = rb.solve(a, b3), O.solve(a, b3)
        assert np.abs(x3 - xo3).max() <= 4 * n * EPS * np.abs(xo3).max() * np.linalg.cond(a, np.inf)


@pytest.mark.parametrize("n", [1, 2, 33, 100, 192])
def test_small_lu_solve_is_the_oracles_bits(rb, n):
    """lu_solve from rustymath's column-major factors (Lu.solve, factor.rs:633-641) up to n = 192:
    with one right-hand side the oracle's lu_solve bit for bit, with three within n*eps of it;
    the transposed solve keeps the block-chained kernels."""
    rng = np.random.default_rng(70 + n)
    a = rng.standard_normal((n, n)) + n * np.eye(n)
    f, p = rb.lu(a)
    b = rng.standard_normal((n, 1))
    assert np.array_equal(rb.lu_solve(f, p, b), O.lu_solve(f, p, b))
    b3 = rng.standard_normal((n, 3))
    x3, xo3 = rb.lu_solve(f, p, b3), O.lu_solve(f, p, b3)
    assert np.abs(x3 - xo3).max() <= 4 * n * EPS * np.abs(xo3).max() * np.linalg.cond(a, np.inf)
    xt = rb.lu_solve(f, p, b3, trans=True)
    assert np.abs(a.T @ xt - b3).max() <= 4 * n * EPS * np.abs(a).sum(0).max() * np.abs(xt).max() + 1e-300


@pytest.mark.parametrize("n", [1, 5, 33, 71, 530])
def test_lu_solve_residuals(rb, n):
    """tests/linalg.rs:384-390: solve and inverse residuals below 4*eps*n."""
    bound = 4 * EPS * max(n, 1)
    a = ref_random(n, n, n + 1)
    fac = rb.lu(a)
    for k in [1, 3]:
        b = ref_random(n, k, 99)
        x = fac.solve(b)
        assert distance(product(a, x), b, max(norm(a) * norm(x), 1.0)) < bound
    inv = fac.inverse()
    assert distance(product(a, inv), np.eye(n), max(norm(a) * norm(inv), 1.0)) < bound


def test_hard_matrices_scaling(rb):
    """tests/linalg.rs:466-483: a power-of-two scaling scales U, the solves and the inverse
    exactly, with the same permutation."""
    n = 40
    tiny = np.finfo(np.float64).tiny / EPS
    quartic = 2.0 ** (int(np.log2(np.finfo(np.float64).max) / 4.0) + 6)
    a, b = ref_random(n, n, 17), ref_random(n, 3, 19)
    f = rb.lu(a)
    for s in [tiny, 1.0 / tiny, quartic]:
        g = rb.lu(a * s)
        assert np.array_equal(g.p, f.p)
        i, j = np.indices((n, n))
        assert np.array_equal(g.factors, np.where(j <= i, f.factors * s, f.factors))
        assert np.array_equal(g.solve(b * s), f.solve(b))
        assert np.array_equal(g.inverse() * s, f.inverse())


@pytest.mark.parametrize("zero", [0, 35, 70])
def test_zero_column(rb, zero):
    """tests/linalg.rs:501-508: finite factors with a zero pivot."""
    n = 71
    a = ref_random(n, n, 29)
    a[:, zero] = 0.0
    f, p = rb.lu(a)
    assert np.isfinite(f).all() and (np.diag(f) == 0.0).any()
    assert distance(product(lower_of(f), upper_of(f)), a[p], norm(a)) < 4 * EPS * n
    with pytest.raises(rb.NotRegular):
        rb.solve(a, np.ones(n))


def test_known_answers(rb):
    """tests/linalg.rs:510-511, 548-558: subnormal pivot, determinants, singular matrices."""
    tiny = np.finfo(np.float64).tiny
    p, q = tiny / 1024.0, tiny / 1048576.0
    f, _ = rb.lu(np.array([[p, 1.0], [q, 1.0]]))
    assert f.reshape(-1).tolist() == [p, q / p, 1.0, 1.0 - q / p]
    swapped = np.array([0., 2, 0, 0, 1, 0, 0, 0, 0, 0, 3, 0, 0, 0, 0, 4]).reshape(4, 4)
    assert rb.lu(swapped).determinant() == -24.0
    singular = np.array([[1.0, 0.0], [3.0, 0.0]])
    assert rb.lu(singular).determinant() == 0.0
    assert rb.lu(singular).log_determinant() == (0.0, -np.inf)
    with pytest.raises(rb.NotRegular):
        rb.solve(np.array([[1.0, 2.0], [2.0, 4.0]]), np.ones(2))


def test_nan_pivot_column(rb):
    """A column of NaN: the pivot rule never picks NaN and keeps the diagonal (factor.rs:476)."""
    a = ref_random(20, 20, 3)
    a[5:, 5] = np.nan
    f, p = rb.lu(a)
    fo, po = O.lu_factor(a)
    assert np.array_equal(p, po)


# ---------------------------------------------------------------- solve

def test_solve_config_small(rb):
    """The n=512, nrhs=1 system (A = N(0,1) + 512 I, b = N(0,1), default_rng(0)): within
    n*eps of the oracle's solution, with backward error <= n * 2^-53."""
    n = 512
    rng = np.random.default_rng(0)
    a = rng.standard_normal((n, n)) + n * np.eye(n)
    b = rng.standard_normal(n)
    x, reps = rb.solve_report(a, b)
    xo = O.solve(a, b)
    assert np.abs(x - xo).max() / np.abs(xo).max() <= n * EPS
    assert O.backward_error(a, x, b) <= n * 2.0 ** -53
    assert reps[0].backward_error <= n * 2.0 ** -53


def test_matmul_config_small(rb):
    """The 512^3 product with U(-1,1) entries, default_rng(0): |error| <= 2k eps |A||B|."""
    rng = np.random.default_rng(0)
    a, b = rng.uniform(-1, 1, (512, 512)), rng.uniform(-1, 1, (512, 512))
    got = rb.matmul(a, b)
    want = O.dgemm(a, b)
    assert (np.abs(got - want) <= 2 * 512 * EPS * (np.abs(a) @ np.abs(b))).all()


@pytest.mark.parametrize("n,k", [(1, 1), (3, 2), (64, 16), (65, 17), (1000, 5), (2048, 16)])
def test_solve_matches_oracle(rb, n, k):
    rng = np.random.default_rng(n + k)
    a = rng.standard_normal((n, n)) + n * np.eye(n)
    b = rng.standard_normal((n, k))
    x = rb.solve(a, b)
    xo = O.solve(a, b)
    assert np.abs(x - xo).max() / np.abs(xo).max() <= n * EPS
    assert O.backward_error(a, x, b) <= n * 2.0 ** -53


def test_lu_solve_transposed(rb):
    n, k = 200, 3
    a = ref_random(n, n, 8) + 3 * np.eye(n)
    b = ref_random(n, k, 9)
    fac = rb.lu(a)
    x = rb.lu_solve(fac.factors, fac.p, b, trans=True)
    xo = O.lu_solve_transposed(*O.lu_factor(a), b)
    assert np.abs(x - xo).max() <= 1e3 * n * EPS * np.abs(xo).max()


def test_python_lu_stack(rb):
    """tests/test_linalg.py:6-32 at float64: the base-matrix stack against NumPy."""
    base = np.array([[0., 2, 1], [3, 1, -1], [1, 0, 4]])
    b = np.arange(12.).reshape(3, 4)[:, ::-1]
    a = np.stack([base + k / 8 * np.eye(3) for k in range(64)])
    f = rb.lu(a)
    assert f.factors.dtype == np.float64 and f.p.dtype == np.int64
    assert np.allclose(f.l @ f.u, np.take_along_axis(a, f.p[..., :, None], -2))
    assert np.allclose(rb.solve(a, np.broadcast_to(b, (64, 3, 4))), np.linalg.solve(a, b))
    assert np.allclose(f.inverse(), np.linalg.inv(a))
    assert np.allclose(f.determinant(), np.linalg.det(a))
    sign, log = f.log_determinant()
    want = np.linalg.slogdet(a)
    assert np.allclose(sign, want.sign) and np.allclose(log, want.logabsdet)
    with pytest.raises(IndexError):
        rb.Lu(rb.lu(base).factors, np.array([-1, 0, 1])).solve(b)


def test_frames_pair_from_the_front(rb):
    """tests/test_linalg.py:94-104: frames pair from the front, unlike NumPy."""
    rng = np.random.default_rng(0)
    a, b = rng.standard_normal((4, 5, 5)), rng.standard_normal((4, 5, 3))
    v = b[0, :, 0]
    assert np.allclose(rb.solve(a, b), np.linalg.solve(a, b))
    assert np.allclose(rb.solve(a[0], v), np.linalg.solve(a[0], v))
    c = rng.standard_normal((4, 2, 5, 3))
    assert np.allclose(rb.solve(a, c), np.linalg.solve(a[:, None], c))
    assert np.allclose(rb.matmul(a, b), a @ b) and np.allclose(rb.matmul(a[0], v), a[0] @ v)


def test_device_tensors(rb):
    """torch CUDA tensors run on the current stream and give tensors back."""
    import torch
    n = 300
    rng = np.random.default_rng(1)
    a = rng.standard_normal((n, n)) + n * np.eye(n)
    b = rng.standard_normal((n, 4))
    ta, tb = torch.tensor(a, device="cuda"), torch.tensor(b, device="cuda")
    x = rb.solve(ta, tb)
    assert x.is_cuda and x.dtype == torch.float64
    assert np.allclose(x.cpu().numpy(), O.solve(a, b), rtol=0, atol=n * EPS * 10)
    fac = rb.lu(ta)
    fo, po = O.lu_factor(a)
    assert np.array_equal(fac.p.cpu().numpy(), po)
    c = rb.matmul(ta, tb)
    assert np.allclose(c.cpu().numpy(), a @ b, rtol=1e-13, atol=1e-12)


@pytest.mark.parametrize("k", [1, 5, 16, 17, 40])
def test_backward_error_report(rb, k):
    """The device's FP64 backward error agrees with the oracle's double-double one."""
    n = 700
    rng = np.random.default_rng(k)
    a = rng.standard_normal((n, n)) + np.sqrt(n) * np.eye(n)
    b = rng.standard_normal((n, k))
    x, reps = rb.solve_report(a, b)
    want = O.backward_error(a, x, b)
    got = reps[0].backward_error
    assert got <= n * 2.0 ** -53 and want <= n * 2.0 ** -53
    assert abs(got - want) <= 4 * EPS * max(1.0, np.sqrt(n)) + 0.5 * want
