"""Parity at the benchmarked configurations, against the oracle (rustymath's algorithms
restated in C), on the same inputs the benchmark builds (bench.make_system, bench.make_batch):

- the single large system, n = 8192 with 16 right-hand sides and kappa = 1e4: both methods
  within kappa n eps (normwise, relative) of the oracle's solution, at normwise backward error
  <= n 2^-53 by the oracle's double-double residual, and the plain float64 LU no farther from
  the oracle than 4 times a third float64 LU (LAPACK getrf + getrs) is. At this kappa two
  backward-stable float64 solves with different rounding orders differ by about kappa times
  their backward errors (measured: 9e-12, against n eps = 1.8e-12), so n eps is not a bar any
  float64 LU other than the oracle's own operation order can meet here; the batched
  configuration below (kappa < 10) is held to n eps;
- 20,000 uneven systems (n ~ U{8..256}, A = N(0,1) + n I): a seeded sample of 500 systems,
  the plain method within n eps of the oracle, the mixed one within kappa_inf n eps, and every
  sampled system's backward error <= n 2^-53;
- the float64 matmul at 2048^3 on wide-range inputs: rm_dgemm and the Ozaki product (8
  slices) against the oracle's PlusTimes product, each item within n eps (|A||B|)_ij."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu
EPS = np.finfo(np.float64).eps


@pytest.fixture(scope="module")
def rb():
    import rustymath_b200 as rb
    return rb


def _fwd(x, xo):
    """max over columns of ||x_c - xo_c||inf / ||xo_c||inf"""
    return float((np.abs(x - xo).max(0) / np.abs(xo).max(0)).max())


def test_single_large_system_matches_the_oracle(rb):
    import os
    import torch
    from bench import make_system
    n, k = 8192, 16
    a, b = make_system(n, k, 0, "cuda")
    a_h, b_h = a.cpu().numpy(), b.cpu().numpy()
    O.set_threads(os.cpu_count())
    xo = O.solve(a_h, b_h)
    x_plain = rb.solve(a, b, method="plain").cpu().numpy()
    x_mixed, reps = rb.solve_report(a, b, method="mixed")
    x_mixed = x_mixed.cpu().numpy()
    assert reps[0].fell_back == 0 and reps[0].method_used == 1
    import scipy.linalg as sl
    lapack = sl.lu_solve(sl.lu_factor(a_h, check_finite=False), b_h, check_finite=False)
    assert _fwd(x_plain, xo) <= 1e4 * n * EPS
    assert _fwd(x_plain, xo) <= 4 * _fwd(lapack, xo)
    assert _fwd(x_mixed, xo) <= 1e4 * n * EPS
    assert O.backward_error(a_h, x_plain, b_h) <= n * 2.0 ** -53
    assert O.backward_error(a_h, x_mixed, b_h) <= n * 2.0 ** -53
    del a, b
    torch.cuda.empty_cache()


def test_batched_configuration_sample_matches_the_oracle(rb):
    import torch
    from bench import make_batch
    ns, ks, a, b = make_batch(20000, 1, "cuda")
    a_off = np.concatenate([[0], np.cumsum(ns * ns)[:-1]])
    b_off = np.concatenate([[0], np.cumsum(ns * ks)[:-1]])
    xs = {}
    for method in ("plain", "mixed"):
        x = torch.zeros(int((ns * ks).sum()), dtype=torch.float64, device="cuda")
        plan = rb.BatchPlan(ns, ks, method=method)
        plan.execute(a, b, x)
        rep = plan.results()[3]
        assert rep.fell_back == 0 and rep.not_regular == 0
        assert rep.max_backward_error <= 256 * 2.0 ** -53
        xs[method] = x.cpu().numpy()
        plan.close()
    a_h, b_h = a.cpu().numpy(), b.cpu().numpy()
    O.set_threads(1)
    for i in np.sort(np.random.default_rng(0).choice(len(ns), 500, replace=False)):
        n, k = int(ns[i]), int(ks[i])
        ai = a_h[a_off[i]:a_off[i] + n * n].reshape(n, n)
        bi = b_h[b_off[i]:b_off[i] + n * k].reshape(n, k)
        xo = O.solve(ai, bi)
        kappa = np.linalg.cond(ai, np.inf)
        xp = xs["plain"][b_off[i]:b_off[i] + n * k].reshape(n, k)
        xm = xs["mixed"][b_off[i]:b_off[i] + n * k].reshape(n, k)
        assert _fwd(xp, xo) <= n * EPS, (i, n)
        assert _fwd(xm, xo) <= kappa * n * EPS, (i, n)
        assert O.backward_error(ai, xp, bi) <= n * 2.0 ** -53
        assert O.backward_error(ai, xm, bi) <= n * 2.0 ** -53


def test_matmul_2048_matches_the_oracle(rb):
    import os
    import torch
    n = 2048
    rng = np.random.default_rng(5)
    a = rng.uniform(-1, 1, (n, n)) * 10.0 ** rng.uniform(-3, 3, (n, 1))
    b = rng.uniform(-1, 1, (n, n)) * 10.0 ** rng.uniform(-3, 3, (1, n))
    O.set_threads(os.cpu_count())
    ref = O.dgemm(a, b)
    mag = np.abs(a) @ np.abs(b)
    ta, tb = torch.tensor(a, device="cuda"), torch.tensor(b, device="cuda")
    native = rb.matmul(ta, tb).cpu().numpy()
    ozaki = rb.linalg.matmul_ozaki(ta, tb, slices=8).cpu().numpy()
    assert (np.abs(native - ref) <= n * EPS * mag).all()
    assert (np.abs(ozaki - ref) <= n * EPS * mag).all()
