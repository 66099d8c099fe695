"""Batched solves of uneven systems (rm_dsolve_batched / rm_batch_plan_*), checked system by
system against the oracle: the normwise backward error (double-double residual) must be at
most n * 2^-53 for the mixed method, and the plain float64 method must agree with the
oracle's solve within the forward error kappa * n * eps allows."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu
EPS = np.finfo(np.float64).eps
EDGE = [1, 2, 3, 8, 15, 16, 17, 31, 32, 33, 63, 64, 65, 127, 128, 129, 191, 192, 193, 255, 256]


@pytest.fixture(scope="module")
def rb():
    import rustymath_b200 as rb
    return rb


def shifted(n, k, seed):
    """The batched configuration's systems: A = N(0,1) + n I, B = N(0,1)."""
    rng = np.random.default_rng(seed)
    return rng.standard_normal((n, n)) + n * np.eye(n), rng.standard_normal((n, k))


def general(n, k, seed):
    """N(0,1) matrices: row exchanges matter."""
    rng = np.random.default_rng(seed)
    return rng.standard_normal((n, n)), rng.standard_normal((n, k))


def batch(sizes, ks, make, seed=0):
    As, Bs = [], []
    for i, (n, k) in enumerate(zip(sizes, ks)):
        a, b = make(n, k, seed + i)
        As.append(a)
        Bs.append(b)
    return As, Bs


def check_bar(As, Bs, Xs):
    for a, b, x in zip(As, Bs, Xs):
        n = a.shape[0]
        assert O.backward_error(a, x, b) <= max(n, 1) * 2.0 ** -53, n


def test_mixed_uneven_edges(rb):
    rng = np.random.default_rng(1)
    sizes = EDGE + list(rng.integers(8, 257, 60))
    ks = list(rng.integers(1, 9, len(sizes)))
    As, Bs = batch(sizes, ks, shifted)
    Xs, rep = rb.solve_batched(As, Bs, method="mixed")
    check_bar(As, Bs, Xs)
    assert rep.fell_back == 0 and rep.not_regular == 0
    assert rep.max_backward_error <= 256 * 2.0 ** -53
    assert 1 <= rep.max_iterations <= 3


def test_mixed_general_matrices_need_pivots(rb):
    rng = np.random.default_rng(2)
    sizes = [5, 33, 100, 200, 256, 129, 64]
    As, Bs = batch(sizes, [3] * len(sizes), general, seed=10)
    Xs, rep = rb.solve_batched(As, Bs, method="mixed")
    check_bar(As, Bs, Xs)
    for a, b, x in zip(As, Bs, Xs):
        xo = O.solve(a, b)
        kappa = np.linalg.cond(a)
        assert np.abs(x - xo).max() <= kappa * a.shape[0] * EPS * np.abs(xo).max()


def test_plain_matches_oracle(rb):
    sizes = [1, 7, 32, 90, 256, 150]
    As, Bs = batch(sizes, [2, 1, 8, 4, 3, 5], general, seed=20)
    Xs, rep = rb.solve_batched(As, Bs, method="plain")
    assert rep.fell_back == 0 and rep.max_iterations == 0
    for a, b, x in zip(As, Bs, Xs):
        xo = O.solve(a, b)
        kappa = np.linalg.cond(a)
        assert np.abs(x - xo).max() <= kappa * a.shape[0] * EPS * np.abs(xo).max()
    check_bar(As, Bs, Xs)


def test_stall_falls_back_and_singular_is_flagged(rb):
    from rustymath_b200 import _lib
    n = 120
    rng = np.random.default_rng(3)
    u, _ = np.linalg.qr(rng.standard_normal((n, n)))
    v, _ = np.linalg.qr(rng.standard_normal((n, n)))
    hard = (u * np.logspace(0, -12, n)) @ v.T  # beyond float32 factors' reach
    As = [shifted(40, 2, 4)[0], hard, np.ones((9, 9)), shifted(200, 1, 5)[0]]
    Bs = [rng.standard_normal((40, 2)), rng.standard_normal((n, 3)), np.ones((9, 1)), rng.standard_normal((200, 1))]
    plan = rb.BatchPlan([a.shape[0] for a in As], [b.shape[1] for b in Bs], method="mixed")
    a, b = plan.pack(As, Bs, device="cuda")
    import torch
    x = torch.zeros(plan.b_size, dtype=torch.float64, device="cuda")
    plan.execute(a, b, x)
    berr, iters, flags, rep = plan.results()
    Xs = [t.cpu().numpy() for t in plan.unpack(x)]
    assert flags[0] == 0 and flags[3] == 0
    assert flags[1] & _lib.RM_BATCH_FELL_BACK and not flags[1] & _lib.RM_BATCH_NOT_REGULAR
    assert flags[2] & _lib.RM_BATCH_NOT_REGULAR
    assert rep.fell_back == 2 and rep.not_regular == 1
    for i in (0, 1, 3):
        assert O.backward_error(As[i], Xs[i], Bs[i]) <= As[i].shape[0] * 2.0 ** -53
    plan.close()


def test_empty_systems_and_empty_batch(rb):
    As = [np.zeros((0, 0)), shifted(10, 1, 6)[0], np.zeros((0, 0))]
    Bs = [np.zeros((0, 1)), np.ones((10, 1)), np.zeros((0, 2))]
    Xs, rep = rb.solve_batched(As, Bs)
    assert Xs[0].shape == (0, 1) and Xs[2].shape == (0, 2)
    check_bar(As[1:2], Bs[1:2], Xs[1:2])
    Xs, rep = rb.solve_batched([], [])
    assert Xs == []


def test_too_large_is_rejected(rb):
    with pytest.raises(ValueError):
        rb.BatchPlan([257], [1])
    with pytest.raises(ValueError):
        rb.BatchPlan([10], [9])


def test_tune_and_graph_replay(rb):
    import torch
    rng = np.random.default_rng(7)
    sizes = list(rng.integers(8, 257, 300))
    ks = list(rng.integers(1, 5, 300))
    As, Bs = batch(sizes, ks, shifted, seed=100)
    plan = rb.BatchPlan(sizes, ks, method="mixed")
    a, b = plan.pack(As, Bs, device="cuda")
    x = torch.zeros(plan.b_size, dtype=torch.float64, device="cuda")
    assert plan.cta_threads() == [64, 64, 256, 256, 256]
    widths = plan.tune(a, b, x)
    assert all(w in (16, 32) for w in widths)
    threads = plan.cta_threads()
    assert threads[2:] == [256] * 3 and all(t in (64, 256) for t in threads[:2])
    assert threads[0] == 64 or threads[1] == 256  # one split of the size-sorted order
    # the tuner's last trial ran the systems of n <= 64 on 256-thread CTAs
    check_bar(As, Bs, [t.cpu().numpy() for t in plan.unpack(x)])
    plan.execute(a, b, x)
    check_bar(As, Bs, [t.cpu().numpy() for t in plan.unpack(x)])
    # the same pointers replay the captured graph; new right-hand sides in place
    Bs2 = [rng.standard_normal(bb.shape) for bb in Bs]
    _, b2 = plan.pack(As, Bs2, device="cuda")
    b.copy_(b2)
    plan.execute(a, b, x)
    torch.cuda.synchronize()
    check_bar(As, Bs2, [t.cpu().numpy() for t in plan.unpack(x)])
    # new pointers capture again
    x2 = torch.zeros_like(x)
    plan.execute(a, b, x2)
    torch.cuda.synchronize()
    assert torch.equal(x, x2)
    plan.close()


def test_tune_precision(rb):
    """The tuner's precision axis: every size bucket keeps float32 factors + refinement or takes
    float64 factors, whichever it timed faster; either way every system meets n 2^-53, the
    float64 route's systems report no refinement steps, and the adjoint follows each system's
    factors. A plain plan has no choice to make."""
    import torch
    rng = np.random.default_rng(11)
    sizes = list(rng.integers(8, 257, 200)) + [1, 256]
    ks = list(rng.integers(1, 5, 202))
    As, Bs = batch(sizes, ks, shifted, seed=300)
    plan = rb.BatchPlan(sizes, ks, method="mixed")
    a, b = plan.pack(As, Bs, device="cuda")
    x = torch.zeros(plan.b_size, dtype=torch.float64, device="cuda")
    assert plan.precision() == ["mixed"] * 5
    plan.tune(a, b, x, precision=True)
    routes = plan.precision()
    assert all(r in ("mixed", "plain") for r in routes)
    plan.execute(a, b, x)
    torch.cuda.synchronize()
    Xs = [t.cpu().numpy() for t in plan.unpack(x)]
    check_bar(As, Bs, Xs)
    berr, iters, flags, rep = plan.results()
    bounds = [32, 64, 128, 192, 256]
    for n, it in zip(sizes, iters):
        if routes[next(i for i, m in enumerate(bounds) if n <= m)] == "plain":
            assert it == 0
    assert rep.fell_back == 0
    # the adjoint reads each system's own factor type
    gx = torch.randn(plan.b_size, dtype=torch.float64, device="cuda", generator=torch.Generator("cuda").manual_seed(1))
    gb = torch.empty_like(gx)
    plan.adjoint(a, x, gx, gb)
    torch.cuda.synchronize()
    for aa, g, y in zip(As, plan.unpack(gx), plan.unpack(gb)):
        yo = np.linalg.solve(aa.T, g.cpu().numpy())
        assert np.abs(y.cpu().numpy() - yo).max() <= 1e-12 * max(1.0, np.abs(yo).max())
    plan.close()
    plain = rb.BatchPlan(sizes, ks, method="plain")
    plain.tune(a, b, x, precision=True)
    assert plain.precision() == ["plain"] * 5
    plain.close()


def test_device_lists(rb):
    import torch
    As, Bs = batch([50, 130], [2, 1], shifted, seed=30)
    ta = [torch.tensor(a, device="cuda") for a in As]
    tb = [torch.tensor(b[:, 0], device="cuda") if b.shape[1] == 1 else torch.tensor(b, device="cuda") for b in Bs]
    Xs, rep = rb.solve_batched(ta, tb)
    assert Xs[1].shape == (130,) and Xs[1].is_cuda
    check_bar(As, Bs, [Xs[0].cpu().numpy(), Xs[1].cpu().numpy().reshape(-1, 1)])


def test_host_form(rb):
    import ctypes
    from rustymath_b200 import _lib
    sizes, ks = [12, 100, 3], [2, 1, 4]
    As, Bs = batch(sizes, ks, general, seed=40)
    plan_ns, plan_ks = np.array(sizes, np.int64), np.array(ks, np.int64)
    a_off = np.array([0, 144, 144 + 10000], np.int64)
    b_off = np.array([0, 24, 124], np.int64)
    a = np.concatenate([x.ravel() for x in As])
    b = np.concatenate([x.ravel() for x in Bs])
    x = np.zeros_like(b)
    rep = _lib.BatchReport()
    opts = rb.linalg._options("mixed")
    st = _lib.load().rm_dsolve_batched_host(3, plan_ns.ctypes.data, plan_ks.ctypes.data, a_off.ctypes.data,
                                            b_off.ctypes.data, b_off.ctypes.data, a.ctypes.data, b.ctypes.data,
                                            x.ctypes.data, ctypes.byref(opts), ctypes.byref(rep))
    _lib.check(st, "rm_dsolve_batched_host")
    Xs = [x[o:o + n * k].reshape(n, k) for o, n, k in zip(b_off, sizes, ks)]
    check_bar(As, Bs, Xs)


def test_execute_from_host_memory(rb):
    """execute_host (copies in groups that overlap the solves) gives the same bits as execute,
    also after a tune (which may change the panel widths, so both run again), and with offsets
    that do not follow the systems' order (one group)."""
    import torch
    rng = np.random.default_rng(11)
    sizes = list(rng.integers(8, 257, 200)) + [3, 64, 65, 256]
    ks = list(rng.integers(1, 5, len(sizes)))
    As, Bs = batch(sizes, ks, shifted, seed=300)
    plan = rb.BatchPlan(sizes, ks, method="mixed")
    a, b = plan.pack(As, Bs, device="cuda")
    x = torch.zeros(plan.b_size, dtype=torch.float64, device="cuda")
    plan.execute(a, b, x)
    torch.cuda.synchronize()
    want = x.cpu()
    a_h, b_h = a.cpu().pin_memory(), b.cpu().pin_memory()
    x_h = torch.zeros(plan.b_size, dtype=torch.float64).pin_memory()
    a2, b2, x2 = torch.zeros_like(a), torch.zeros_like(b), torch.zeros_like(x)
    plan.execute_host(a_h, b_h, x_h, a2, b2, x2)
    torch.cuda.synchronize()
    assert torch.equal(x_h, want)
    assert plan.results()[3].fell_back == 0
    plan.tune(a, b, x)  # new panel widths (and so other float32 roundings): compare anew
    plan.execute(a, b, x)
    torch.cuda.synchronize()
    want = x.cpu()
    x_h.zero_()
    plan.execute_host(a_h, b_h, x_h, a2, b2, x2)
    torch.cuda.synchronize()
    assert torch.equal(x_h, want)
    check_bar(As, Bs, [t.numpy() for t in plan.unpack(x_h)])
    plan.close()
    # systems packed in reverse order: one group
    from rustymath_b200 import _lib
    import ctypes
    ns = np.array([5, 40, 90], np.int64)
    kk = np.array([1, 2, 3], np.int64)
    a_off = np.array([40 * 40 + 90 * 90, 90 * 90, 0], np.int64)
    b_off = np.array([2 * 40 + 3 * 90, 3 * 90, 0], np.int64)
    As3, Bs3 = batch(list(ns), list(kk), shifted, seed=400)
    a3 = np.zeros(int((ns * ns).sum()))
    b3 = np.zeros(int((ns * kk).sum()))
    for i in range(3):
        a3[a_off[i]:a_off[i] + ns[i] ** 2] = As3[i].ravel()
        b3[b_off[i]:b_off[i] + ns[i] * kk[i]] = Bs3[i].ravel()
    h = ctypes.c_void_p()
    lib = _lib.load()
    _lib.check(lib.rm_batch_plan_create(3, ns.ctypes.data, kk.ctypes.data, a_off.ctypes.data, b_off.ctypes.data,
                                        b_off.ctypes.data, None, ctypes.byref(h)), "plan")
    ah, bh = torch.tensor(a3).pin_memory(), torch.tensor(b3).pin_memory()
    xh = torch.zeros_like(bh).pin_memory()
    ad, bd, xd = torch.zeros(a3.size, dtype=torch.float64, device="cuda"), torch.zeros(b3.size, dtype=torch.float64,
                                                                                        device="cuda"), \
        torch.zeros(b3.size, dtype=torch.float64, device="cuda")
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    _lib.check(lib.rm_batch_plan_execute_host(h, ctypes.c_void_p(ah.data_ptr()), ctypes.c_void_p(bh.data_ptr()),
                                              ctypes.c_void_p(xh.data_ptr()), ctypes.c_void_p(ad.data_ptr()),
                                              ctypes.c_void_p(bd.data_ptr()), ctypes.c_void_p(xd.data_ptr()), s), "ex")
    torch.cuda.synchronize()
    for i in range(3):
        xi = xh.numpy()[b_off[i]:b_off[i] + ns[i] * kk[i]].reshape(ns[i], kk[i])
        assert O.backward_error(As3[i], xi, Bs3[i]) <= ns[i] * 2.0 ** -53
    lib.rm_batch_plan_destroy(h)
