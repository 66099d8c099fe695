"""What an LU gives besides one solve, on the GPU, against the oracle (rustymath's algorithms
restated) and the reference's own known answers:
  - Lu.inverse (rm_dlu_inverse; factor.rs:645-664): residual below 4 eps n (tests/linalg.rs:389),
    within kappa n eps of the oracle's inverse, and exact under power-of-two scaling
    (tests/linalg.rs:482);
  - determinants (rm_dlu_determinant; factor.rs:174-194): -24 and 0 and (0, -inf) exactly
    (tests/linalg.rs:552-558), stacks against the oracle's in-order fold (relative 4 n eps);
  - stacks in one launch: lu (rm_dlu_factor_batched) with the oracle's row positions and
    factors within 1e3 n eps of its, lu_solve (rm_dlu_solve_batched) including the transposed
    form, solve through the batched kernel;
  - rustymath's dtype ladder on results (python/rustymath/linalg.py:1)."""
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


def _launches(rb):
    return rb._lib.load().rm_launch_count()


@pytest.mark.parametrize("n", [1, 2, 5, 31, 32, 33, 71, 130, 530])
def test_inverse_matches_the_oracle(rb, n):
    a = ref_random(n, n, n + 1)
    f = rb.lu(a)
    inv = f.inverse()
    assert distance(O.dgemm(a, inv), np.eye(n), max(norm(a) * norm(inv), 1.0)) < 4 * EPS * max(n, 1)
    fo, po = O.lu_factor(a)
    want = O.lu_inverse(fo, po)
    kappa = np.linalg.cond(a)
    assert np.abs(inv - want).max() <= kappa * n * EPS * np.abs(want).max()


def test_inverse_scaling_is_exact(rb):
    """tests/linalg.rs:478-482: scaling by a power of two s scales the inverse by 1/s exactly."""
    import torch
    n = 40
    a = ref_random(n, n, 17)
    tiny = np.finfo(np.float64).tiny / EPS
    quartic = 2.0 ** (int(np.log2(np.finfo(np.float64).max) / 4.0) + 6)
    base = rb.lu(torch.tensor(a, device="cuda")).inverse()
    for s in [tiny, 1.0 / tiny, quartic]:
        got = rb.lu(torch.tensor(a * s, device="cuda")).inverse()
        assert torch.equal(got * s, base)


def test_known_determinants(rb):
    swapped = np.array([0., 2, 0, 0, 1, 0, 0, 0, 0, 0, 3, 0, 0, 0, 0, 4]).reshape(4, 4)
    assert rb.det(swapped) == -24.0
    singular = np.array([[1.0, 0.0], [3.0, 0.0]])
    assert rb.det(singular) == 0.0
    assert rb.slogdet(singular) == (0.0, -np.inf)
    assert rb.slogdet([[1., 2], [2, 4]]) == (0.0, -np.inf)  # tests/test_linalg.py:182


def test_determinant_stack_matches_the_oracle(rb):
    rng = np.random.default_rng(4)
    n = 37
    stack = rng.standard_normal((12, n, n))
    l0 = _launches(rb)
    f = rb.lu(stack)
    d = f.determinant()
    assert _launches(rb) - l0 == 2  # one batched LU, one determinant launch
    sign, log = f.log_determinant()
    for i in range(12):
        fo, po = O.lu_factor(stack[i])
        assert np.array_equal(f.p[i], po)
        want = O.lu_determinant(fo, po)
        assert abs(d[i] - want) <= 4 * n * EPS * abs(want)
        ws, wl = O.lu_log_determinant(fo, po)
        assert sign[i] == ws and abs(log[i] - wl) <= 4 * n * EPS * max(1.0, abs(wl))
    assert np.allclose(rb.det(stack), np.linalg.det(stack))
    s2, l2 = rb.slogdet(stack)
    want = np.linalg.slogdet(stack)
    # rustymath's sign folds sign * (d * (1/|d|)) (factor.rs:181), which can land an ulp from 1;
    # against the oracle it is exact (above), against NumPy's exact +-1 within a few ulps
    assert np.allclose(s2, want.sign, rtol=0, atol=8 * EPS) and np.allclose(l2, want.logabsdet)


@pytest.mark.parametrize("n", [1, 7, 64, 129, 256])
def test_stacked_lu_is_one_launch_with_the_oracles_pivots(rb, n):
    rng = np.random.default_rng(n)
    stack = rng.standard_normal((20, n, n))
    l0 = _launches(rb)
    f = rb.lu(stack)
    assert _launches(rb) - l0 == 1
    for i in range(20):
        fo, po = O.lu_factor(stack[i])
        assert np.array_equal(f.p[i], po), i
        assert np.abs(f.factors[i] - fo).max() <= 1e3 * n * EPS * np.abs(fo).max()


@pytest.mark.parametrize("trans", [False, True])
def test_stacked_lu_solve(rb, trans):
    import torch
    rng = np.random.default_rng(6)
    n, k = 90, 3
    stack = rng.standard_normal((16, n, n)) + 3 * np.eye(n)
    b = rng.standard_normal((16, n, k))
    f = rb.lu(torch.tensor(stack, device="cuda"))
    x = rb.lu_solve(f.factors, f.p, torch.tensor(b, device="cuda"), trans=trans).cpu().numpy()
    for i in range(16):
        fo, po = O.lu_factor(stack[i])
        want = O.lu_solve_transposed(fo, po, b[i]) if trans else O.lu_solve(fo, po, b[i])
        kappa = np.linalg.cond(stack[i])
        assert np.abs(x[i] - want).max() <= kappa * n * EPS * np.abs(want).max()
    with pytest.raises(IndexError):
        bad = f.p.clone()
        bad[3, 5] = n
        rb.lu_solve(f.factors, bad, torch.tensor(b, device="cuda"))


def test_stacked_solve_is_batched(rb):
    """A 64-stack of 3 x 3 systems (tests/test_linalg.py:6-32) goes through the batched kernel:
    one graph launch, not 64 solves."""
    base = np.array([[0., 2, 1], [3, 1, -1], [1, 0, 4]])
    b = np.arange(12.).reshape(3, 4)[:, ::-1]
    a = np.stack([base + k / 8 * np.eye(3) for k in range(64)])
    l0 = _launches(rb)
    x = rb.solve(a, np.broadcast_to(b, (64, 3, 4)))
    assert _launches(rb) - l0 == 1
    for i in range(64):
        assert np.abs(x[i] - O.solve(a[i], b)).max() <= 3 * EPS * 1e3 * np.abs(x[i]).max()


def test_dtype_ladder(rb):
    """float32 and float64 keep their dtype, float16 results are float16, small integers and
    Booleans give float32, wider integers float64 (python/rustymath/linalg.py:1)."""
    rng = np.random.default_rng(8)
    a = rng.standard_normal((4, 6, 6)) + 6 * np.eye(6)
    b = rng.standard_normal((4, 6, 2))
    for dt, tol in [(np.float32, 1e-5), (np.float16, 2e-2)]:
        x = rb.solve(a.astype(dt), b.astype(dt))
        assert x.dtype == dt
        assert np.allclose(x, np.linalg.solve(a.astype(dt).astype(np.float64), b.astype(dt).astype(np.float64)),
                           rtol=tol, atol=tol)
        assert rb.lu(a.astype(dt)).factors.dtype == dt
        assert rb.det(a.astype(dt)).dtype == dt
    ai = np.array([[4, 1], [2, 3]])
    assert rb.solve(ai.astype(np.int16), np.array([1, 2], np.int16)).dtype == np.float32
    assert rb.solve(ai.astype(np.int64), np.array([1, 2])).dtype == np.float64
    assert np.allclose(rb.solve(ai, np.array([1, 2])), np.linalg.solve(ai, [1, 2]))
    assert rb.lu(ai).p.dtype == np.int64
    with pytest.raises(TypeError):
        rb.solve(ai.astype(np.complex128), np.array([1, 2]))


@pytest.mark.parametrize("n", [8, 33, 160, 256])
def test_dominant_stacks_take_the_oracles_pivots(rb, n):
    """Column diagonally dominant matrices (N(0,1) + 2n I) factor without a pivot search on the
    GPU; partial pivoting chooses their diagonal at every step, so the row positions are the
    identity, as the oracle's, and the factors agree with the oracle's; a stack mixing them with
    general matrices takes both routes in one launch."""
    rng = np.random.default_rng(n + 100)
    stack = rng.standard_normal((10, n, n))
    stack[::2] += 2 * n * np.eye(n)
    f = rb.lu(stack)
    for i in range(10):
        fo, po = O.lu_factor(stack[i])
        assert np.array_equal(f.p[i], po), i
        if i % 2 == 0:
            assert np.array_equal(po, np.arange(n))
        assert np.abs(f.factors[i] - fo).max() <= 1e3 * n * EPS * np.abs(fo).max()
    b = rng.standard_normal((10, n, 3))
    for method in ("plain", "mixed"):
        x = rb.solve(stack, b, method=method)
        for i in range(10):
            assert O.backward_error(stack[i], x[i], b[i]) <= n * 2.0 ** -53
