"""Products with one output row or column (rm_dgemm with m == 1 or n == 1): rustymath's
by_vector case (core/src/linalg.rs:1020-1073), run as HBM streams (csrc/gemv.cu) instead of DMMA
tiles. Against the oracle (which takes by_vector's route for these shapes): elementwise within
2 k eps (|alpha| |op(A)| |op(B)| + |beta| |C|), for every transpose combination, aligned and odd
leading dimensions, a strided vector, beta = 0 over NaN, and the launches each form takes."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu
EPS = np.finfo(np.float64).eps


@pytest.fixture(scope="module")
def rb():
    import rustymath_b200 as rb
    return rb


def _run(rb, ta, tb, m, n, k, alpha=-1.5, beta=0.5, pad_a=0, pad_b=0, nan_c=False, seed=0):
    rng = np.random.default_rng(seed + 7 * m + 13 * n + k)
    ash = (k, m) if ta else (m, k)
    bsh = (n, k) if tb else (k, n)
    a_full = rng.uniform(-1, 1, (ash[0], ash[1] + pad_a))
    b_full = rng.uniform(-1, 1, (bsh[0], bsh[1] + pad_b))
    a, b = a_full[:, :ash[1]], b_full[:, :bsh[1]]
    c = np.full((m, n), np.nan) if nan_c else rng.uniform(-1, 1, (m, n))
    got = c.copy()
    lib = rb._lib.load()
    l0 = lib.rm_launch_count()
    st = lib.rm_dgemm_host(ta, tb, m, n, k, alpha, a_full.ctypes.data, a_full.shape[1], b_full.ctypes.data,
                           b_full.shape[1], beta, got.ctypes.data, n)
    rb._lib.check(st, "dgemm")
    launches = lib.rm_launch_count() - l0
    want = O.dgemm(np.ascontiguousarray(a), np.ascontiguousarray(b), alpha=alpha, beta=beta,
                   c=np.zeros_like(c) if nan_c else c, ta=bool(ta), tb=bool(tb))
    opa = a.T if ta else a
    opb = b.T if tb else b
    bound = 2 * k * EPS * (abs(alpha) * (np.abs(opa) @ np.abs(opb)) + (0 if nan_c else abs(beta) * np.abs(c)))
    assert np.isfinite(got).all()
    assert (np.abs(got - want) <= bound + 1e-300).all(), np.abs(got - want).max()
    return launches


@pytest.mark.parametrize("ta", [0, 1])
@pytest.mark.parametrize("tb", [0, 1])
@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (1, 1, 1000), (300, 1, 7), (1, 300, 7), (1000, 1, 4099),
                                   (1, 1000, 4099), (3, 1, 130), (1, 257, 65)])
def test_vector_products_match_the_oracle(rb, ta, tb, m, n, k):
    _run(rb, ta, tb, m, n, k)


@pytest.mark.parametrize("ta,tb", [(0, 0), (1, 0), (0, 1), (1, 1)])
def test_odd_leading_dimensions_and_beta_zero(rb, ta, tb):
    """Odd leading dimensions (8-byte aligned rows: the scalar loads, or a gathered vector)
    and beta = 0 over a C of NaN (C is not read, as rustymath's scale)."""
    _run(rb, ta, tb, 513, 1, 301, pad_a=3, pad_b=1)
    _run(rb, ta, tb, 1, 513, 301, pad_a=1, pad_b=3)
    _run(rb, ta, tb, 200, 1, 50, beta=0.0, nan_c=True)


def test_launches(rb):
    """The host form copies each operand with its rows padded to an even length, so a one-column
    operand arrives with a stride of 2 and is gathered first."""
    # n == 1, A not transposed, B stored as one contiguous row (tb = 1): one dot launch
    assert _run(rb, 0, 1, 4096, 1, 4096) == 1
    # B not transposed: its column has stride 2 on the device: the gather, then the dots
    assert _run(rb, 0, 0, 4096, 1, 4096) == 2
    # A transposed: a column combination, the k range split over the GPU, then the fold
    assert _run(rb, 1, 1, 4096, 1, 4096) == 2
    # m == 1, B transposed: dots of B's rows with A's row (A transposed: stride 2, gathered)
    assert _run(rb, 0, 1, 1, 4096, 4096) == 1
    assert _run(rb, 1, 1, 1, 4096, 4096) == 2
