"""Reverse-mode differentiation of batched solves: `solve(a, b)` for stacks of systems as a
torch.autograd.Function.

The forward pass is the batched solve (one persistent launch, rustymath_b200.batched); the
backward pass is the hand-written adjoint kernel: for x = A^-1 b and an upstream gradient
g = dL/dx, dL/db = A^-T g (a transposed solve reusing the forward's LU factors and row
order, refined in float64 against A^T) and dL/dA = -(dL/db) x^T (the rank-k outer product,
formed in the same kernel). rustymath's solve has no derivative; the shapes follow its stack
convention (the matrices in the last two axes).
"""
import torch

from .batched import BatchPlan

__all__ = ["solve", "BatchedSolve"]

# Plans (scratch, sorted order, captured graph) by (device, batch, n, k, method): a training
# loop solving systems of one shape reuses its plans instead of building one per forward. A
# forward's factors live in its plan until its graph is freed (backward may run more than once
# on a retained graph), so a plan is leased to one forward's autograd node and comes back to
# the cache when that node is freed; forwards whose nodes are alive at once get plans of their
# own.
_PLANS = {}


class _Lease:
    def __init__(self, key, plan):
        self.key, self.plan = key, plan

    def __del__(self):
        try:
            free = _PLANS.setdefault(self.key, [])
            if len(free) < 4:
                free.append(self.plan)
                return
        except Exception:  # interpreter shutdown: the cache may be gone already
            pass
        self.plan.close()


def _lease(device, batch, n, k, method):
    key = (str(device), batch, n, k, method)
    free = _PLANS.setdefault(key, [])
    return _Lease(key, free.pop() if free else BatchPlan([n] * batch, [k] * batch, method=method))


class BatchedSolve(torch.autograd.Function):
    """x = A^-1 b for a (batch, n, n) float64 CUDA stack and (batch, n, k) right-hand sides."""

    @staticmethod
    def forward(ctx, a, b, method):
        batch, n, _ = a.shape
        k = b.shape[-1]
        lease = _lease(a.device, batch, n, k, method)
        plan = lease.plan
        af = a.detach().contiguous().view(-1)
        bf = b.detach().contiguous().view(-1)
        x = torch.empty(batch * n * k, dtype=torch.float64, device=a.device)
        if batch:
            plan.execute(af, bf, x)
        ctx.shapes = (batch, n, k)
        # the lease (and so the plan's factors) lives with the node; with no gradient wanted it
        # goes back at once
        ctx.lease = lease if (ctx.needs_input_grad[0] or ctx.needs_input_grad[1]) else None
        ctx.save_for_backward(af, x)
        return x.view(batch, n, k)

    @staticmethod
    def backward(ctx, gx):
        af, x = ctx.saved_tensors
        batch, n, k = ctx.shapes
        plan = ctx.lease.plan
        gb = torch.empty(batch * n * k, dtype=torch.float64, device=x.device)
        ga = torch.empty(batch * n * n, dtype=torch.float64, device=x.device) if ctx.needs_input_grad[0] else None
        if batch:
            plan.adjoint(af, x, gx.detach().to(torch.float64).contiguous().view(-1), gb, ga)
        return (None if ga is None else ga.view(batch, n, n)), gb.view(batch, n, k), None


def solve(a, b, method="mixed"):
    """x with a[i] x[i] = b[i] for a stack a (batch, n, n) and b (batch, n, k) or (batch, n),
    float64 CUDA tensors, n <= 256 and k <= 8; differentiable in a and b."""
    if a.ndim != 3 or a.shape[-1] != a.shape[-2]:
        raise ValueError("solve needs a (batch, n, n) stack")
    vector = b.ndim == 2
    bb = b.unsqueeze(-1) if vector else b
    if bb.shape[:2] != a.shape[:2]:
        raise ValueError("b's leading axes must match a's stack and rows")
    x = BatchedSolve.apply(a.to(torch.float64), bb.to(torch.float64), method)
    return x.squeeze(-1) if vector else x
