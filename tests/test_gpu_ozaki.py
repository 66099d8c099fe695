"""The Ozaki split-precision GEMM (rm_dgemm_ozaki): int8 tensor-core slice products summed in
float64. Checked against an extended-precision product (numpy longdouble, 64-bit mantissa on
x86-64) with rows of A and columns of B scaled over a wide exponent range, as the large-GEMM
configuration states, and against the oracle's float64 GEMM."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def wide(m, k, n, seed):
    rng = np.random.default_rng(seed)
    a = rng.uniform(-1, 1, (m, k)) * 10.0 ** rng.uniform(-3, 3, (m, 1))
    b = rng.uniform(-1, 1, (k, n)) * 10.0 ** rng.uniform(-3, 3, (1, n))
    return a, b


def exact(a, b):
    return (a.astype(np.longdouble) @ b.astype(np.longdouble))


def run(a, b, slices):
    import torch
    import rustymath_b200 as rb
    return rb.linalg.matmul_ozaki(torch.tensor(a, device="cuda"), torch.tensor(b, device="cuda"),
                                  slices=slices).cpu().numpy()


@pytest.mark.parametrize("m,k,n", [(128, 128, 128), (200, 300, 150), (1, 1, 1), (257, 1000, 130), (64, 4096, 96)])
def test_eight_slices_reach_float64(m, k, n):
    a, b = wide(m, k, n, m + k + n)
    ref = exact(a, b)
    got = run(a, b, 8)
    scale = (np.abs(a) @ np.abs(b))
    err = np.abs(got.astype(np.longdouble) - ref).astype(np.float64)
    # float64-level: within a few units of the |A||B| rounding scale
    assert (err <= 4 * 2.0 ** -53 * scale * max(1, np.log2(k))).all()
    # and no worse than the oracle's own float64 product, up to a small factor
    o = O.dgemm(a, b) if hasattr(O, "dgemm") else a @ b
    eo = np.abs(np.asarray(o).astype(np.longdouble) - ref).astype(np.float64)
    assert err.max() <= 4 * max(eo.max(), 2.0 ** -53 * scale.max())


@pytest.mark.parametrize("slices", [2, 4, 6])
def test_fewer_slices_bound(slices):
    m, k, n = 160, 512, 140
    a, b = wide(m, k, n, slices)
    ref = exact(a, b)
    got = run(a, b, slices)
    ra = 2.0 ** np.ceil(np.log2(np.abs(a).max(1, keepdims=True)))
    rb_ = 2.0 ** np.ceil(np.log2(np.abs(b).max(0, keepdims=True)))
    bound = 3 * k * 2.0 ** (-7 * slices) * ra * rb_ + 16 * 2.0 ** -53 * (np.abs(a) @ np.abs(b))
    err = np.abs(got.astype(np.longdouble) - ref).astype(np.float64)
    assert (err <= bound).all()


def test_zero_rows_columns_and_k_zero():
    a, b = wide(100, 64, 90, 5)
    a[7] = 0.0
    b[:, 11] = 0.0
    got = run(a, b, 8)
    assert (got[7] == 0).all() and (got[:, 11] == 0).all()
    assert np.allclose(got, a @ b, rtol=1e-13, atol=1e-13 * np.abs(a @ b).max())
    z = run(np.zeros((5, 0)), np.zeros((0, 4)), 8)
    assert (z == 0).all() and z.shape == (5, 4)


def test_host_form():
    from rustymath_b200 import _lib
    a, b = wide(130, 77, 60, 3)
    c = np.zeros((130, 60))
    st = _lib.load().rm_dgemm_ozaki_host(130, 60, 77, a.ctypes.data, 77, b.ctypes.data, 60, c.ctypes.data, 60, 8)
    _lib.check(st, "rm_dgemm_ozaki_host")
    ref = exact(a, b)
    assert (np.abs(c.astype(np.longdouble) - ref).astype(np.float64) <= 4 * 2.0 ** -53 * 7 * (np.abs(a) @ np.abs(b))).all()
