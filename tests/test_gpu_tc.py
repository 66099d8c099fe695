"""The tcgen05 FP32 GEMM (rm_sgemm_tc) against a float64 product of the same float32 inputs.

Bounds: one TF32 pass rounds each input to 11 significant bits, so |error| <= 2^-9 * k *
|A||B|; three passes keep float32-level products, |error| <= 2^-20 * k * |A||B| (the
dropped low*low term and float32 accumulation)."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def run(passes, a, b, c, alpha, beta, transb=True):
    """C = alpha A B^T + beta C with b given n x k (transb) or as its k x n transpose."""
    import torch
    from rustymath_b200 import _lib
    lib = _lib.load()
    m, k = a.shape
    n = b.shape[0]
    bb = b if transb else np.ascontiguousarray(b.T)
    ta, tb = torch.tensor(a, device="cuda"), torch.tensor(bb, device="cuda")
    tc = torch.tensor(c, device="cuda")
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    st = lib.rm_sgemm_tc(passes, int(transb), m, n, k, alpha, ta.data_ptr(), k, tb.data_ptr(), bb.shape[1], beta,
                         tc.data_ptr(), n, s)
    _lib.check(st, "rm_sgemm_tc")
    torch.cuda.synchronize()
    return tc.cpu().numpy()


@pytest.mark.parametrize("transb", [True, False])
@pytest.mark.parametrize("m,n,k", [(128, 128, 32), (64, 64, 8), (129, 130, 33), (300, 257, 100), (1000, 520, 128),
                                   (256, 384, 1024), (1, 1, 1), (7, 200, 5),
                                   (2304, 2200, 96)])  # more tiles than SMs: both accumulators cycle
def test_sgemm_tc_accuracy(m, n, k, transb):
    rng = np.random.default_rng(m + n + k)
    a = rng.uniform(-1, 1, (m, k)).astype(np.float32)
    b = rng.uniform(-1, 1, (n, k)).astype(np.float32)
    c = rng.uniform(-1, 1, (m, n)).astype(np.float32)
    alpha, beta = -1.0, 1.0
    want = beta * c.astype(np.float64) + alpha * (a.astype(np.float64) @ b.astype(np.float64).T)
    scale = (np.abs(a).astype(np.float64) @ np.abs(b).astype(np.float64).T) + np.abs(c)
    e3 = np.abs(run(3, a, b, c, alpha, beta, transb) - want)
    e1 = np.abs(run(1, a, b, c, alpha, beta, transb) - want)
    assert (e3 <= 2.0 ** -20 * max(k, 1) * scale + 1e-30).all()
    assert (e1 <= 2.0 ** -9 * max(k, 1) * scale + 1e-30).all()
    if k >= 32:
        assert e3.max() < e1.max() / 64  # the low parts recover the bits TF32 drops


def test_sgemm_tc_beta_zero_and_unaligned():
    rng = np.random.default_rng(9)
    m, n, k = 70, 90, 37  # odd k: the operands are copied to padded, aligned buffers
    a = rng.standard_normal((m, k)).astype(np.float32)
    b = rng.standard_normal((n, k)).astype(np.float32)
    c = np.full((m, n), np.nan, np.float32)  # beta = 0 never reads C
    got = run(3, a, b, c, 2.0, 0.0)
    assert np.allclose(got, 2.0 * (a.astype(np.float64) @ b.astype(np.float64).T), rtol=1e-5, atol=1e-5)
    got = run(3, a, b, c, 2.0, 0.0, transb=False)
    want = 2.0 * (a.astype(np.float64) @ b.astype(np.float64).T)
    assert np.allclose(got, want, rtol=1e-5, atol=1e-5)
