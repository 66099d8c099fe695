"""The adjoint of the batched solve (rm_batch_plan_adjoint behind rustymath_b200.autograd):
gradients of L = sum(w * x), x = A^-1 b, against the ones formed from the oracle's solve
(dL/db = A^-T w, dL/dA = -dL/db x^T) and against float64 central finite differences."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def config(batch, n, k, seed):
    """The differentiation configuration's systems: A = N(0,1)/8 + I, b, w ~ N(0,1)."""
    rng = np.random.default_rng(seed)
    a = rng.standard_normal((batch, n, n)) / 8 + np.eye(n)
    b = rng.standard_normal((batch, n, k))
    w = rng.standard_normal((batch, n, k))
    return a, b, w


def grads(a, b, w, method):
    import torch
    from rustymath_b200 import autograd
    ta = torch.tensor(a, device="cuda", requires_grad=True)
    tb = torch.tensor(b, device="cuda", requires_grad=True)
    x = autograd.solve(ta, tb, method=method)
    (x * torch.tensor(w, device="cuda")).sum().backward()
    return x.detach().cpu().numpy(), ta.grad.cpu().numpy(), tb.grad.cpu().numpy()


@pytest.mark.parametrize("method", ["mixed", "plain"])
def test_adjoint_matches_the_oracle(method):
    a, b, w = config(64, 64, 2, 0)
    x, ga, gb = grads(a, b, w, method)
    for i in range(a.shape[0]):
        xo = O.solve(a[i], b[i])
        gbo = O.solve(np.ascontiguousarray(a[i].T), w[i])
        gao = -gbo @ xo.T
        assert np.abs(gb[i] - gbo).max() <= 1e-12 * np.abs(gbo).max()
        assert np.abs(ga[i] - gao).max() <= 1e-12 * np.abs(gao).max()


def test_adjoint_matches_finite_differences():
    """Central differences, h = 1e-6, on random directions of A and b (float64, the oracle's
    solve), against <dL/dA, E_A> + <dL/db, E_b>: 1e-6 relative."""
    a, b, w = config(8, 64, 2, 1)
    _, ga, gb = grads(a, b, w, "mixed")
    rng = np.random.default_rng(2)
    h = 1e-6
    for i in range(a.shape[0]):
        ea = rng.standard_normal(a[i].shape)
        eb = rng.standard_normal(b[i].shape)
        lp = (w[i] * O.solve(a[i] + h * ea, b[i] + h * eb)).sum()
        lm = (w[i] * O.solve(a[i] - h * ea, b[i] - h * eb)).sum()
        fd = (lp - lm) / (2 * h)
        an = (ga[i] * ea).sum() + (gb[i] * eb).sum()
        assert abs(fd - an) <= 1e-6 * max(abs(an), 1.0)


def test_adjoint_uneven_and_fallback():
    import torch
    import rustymath_b200 as rb
    rng = np.random.default_rng(3)
    n_hard = 90
    u, _ = np.linalg.qr(rng.standard_normal((n_hard, n_hard)))
    v, _ = np.linalg.qr(rng.standard_normal((n_hard, n_hard)))
    As = [rng.standard_normal((n, n)) / 8 + np.eye(n) for n in (1, 17, 64, 200)]
    As.append((u * np.logspace(0, -12, n_hard)) @ v.T)  # the float64 fallback's factors
    ks = [1, 3, 2, 8, 2]
    Bs = [rng.standard_normal((a.shape[0], k)) for a, k in zip(As, ks)]
    Gs = [rng.standard_normal(bb.shape) for bb in Bs]
    plan = rb.BatchPlan([a.shape[0] for a in As], ks, method="mixed")
    a, b = plan.pack(As, Bs, device="cuda")
    _, g = plan.pack(As, Gs, device="cuda")
    x = torch.zeros(plan.b_size, dtype=torch.float64, device="cuda")
    plan.execute(a, b, x)
    gb = torch.zeros_like(x)
    ga = torch.zeros(plan.a_size, dtype=torch.float64, device="cuda")
    plan.adjoint(a, x, g, gb, ga)
    berr, mx = plan.adjoint_results()
    xs = [t.cpu().numpy() for t in plan.unpack(x)]
    gbs = [t.cpu().numpy() for t in plan.unpack(gb)]
    offs = np.concatenate([[0], np.cumsum([aa.size for aa in As])])
    for i, (aa, bb, gg) in enumerate(zip(As, Bs, Gs)):
        nn = aa.shape[0]
        assert berr[i] <= nn * 2.0 ** -53
        gbo = O.solve(np.ascontiguousarray(aa.T), gg)
        kappa = np.linalg.cond(aa)
        assert np.abs(gbs[i] - gbo).max() <= kappa * nn * 2.2e-16 * np.abs(gbo).max()
        gai = ga[offs[i]:offs[i + 1]].view(nn, nn).cpu().numpy()
        assert np.allclose(gai, -gbs[i] @ xs[i].T, rtol=1e-13, atol=1e-13 * np.abs(gai).max())
    plan.close()


def test_gradcheck_small():
    import torch
    from rustymath_b200 import autograd
    rng = np.random.default_rng(4)
    a = torch.tensor(rng.standard_normal((3, 5, 5)) + 3 * np.eye(5), device="cuda", requires_grad=True)
    b = torch.tensor(rng.standard_normal((3, 5, 2)), device="cuda", requires_grad=True)
    assert torch.autograd.gradcheck(lambda a, b: autograd.solve(a, b, method="plain"), (a, b), eps=1e-6,
                                    atol=1e-7, rtol=1e-6)


def test_plans_are_reused_across_steps():
    """A training loop of one shape builds its batch plan once (the plan cache), and each
    step's gradients stay right."""
    import torch
    from rustymath_b200 import autograd
    batch, n, k = 32, 20, 2
    g = torch.Generator(device="cuda")
    g.manual_seed(3)
    autograd._PLANS.clear()
    for step in range(3):
        a = (torch.randn(batch, n, n, generator=g, device="cuda", dtype=torch.float64) / 8
             + torch.eye(n, device="cuda", dtype=torch.float64)).requires_grad_()
        b = torch.randn(batch, n, k, generator=g, device="cuda", dtype=torch.float64).requires_grad_()
        x = autograd.solve(a, b)
        x.sum().backward()
        want_b = torch.linalg.solve(a.detach().transpose(-1, -2), torch.ones_like(b))
        assert torch.allclose(b.grad, want_b, rtol=1e-12, atol=1e-12)
        assert torch.allclose(a.grad, -want_b @ x.detach().transpose(-1, -2), rtol=1e-11, atol=1e-11)
        del x  # the step's graph goes, and its plan back to the cache
    plans = [p for free in autograd._PLANS.values() for p in free]
    assert len(plans) == 1
