"""
Differentiable equilibrium: u*(theta) as a torch.autograd.Function whose backward is the adjoint.

    u = equilibrium(theta, params, **solver_options)      forward: device Newton-Krylov solve
                                                          (adjoint_rtol, adjoint_max_iter,
                                                          adjoint_preconditioner and adjoint_on_failure
                                                          configure the backward)
    L = compliance(theta, params, **solver_options)       f . u*(theta)
    L.backward()                                          theta.grad = dL/dtheta by the adjoint kernels

The backward pass receives dL/du*, solves A^T lambda = m * dL/du* with the device PCG at u* and returns
-lambda^T dR/dtheta from the per-element sensitivity kernel.  No graph of the Newton iterations is
recorded.  The adjoint preconditioner defaults to "auto" (geometric multigrid on structured meshes, where
Jacobi would need thousands of iterations at 1e-10; Jacobi otherwise), and an adjoint that stops short of
its tolerance is reported: a warning by default, an error with adjoint_on_failure="raise".  (The reference removed its class-based autograd bridge in favour of compute_sensitivity,
adjoint.py:18-20; this restores the torch.autograd interface on top of the same mathematics.)
"""
import torch

from difffea_b200.adjoint import compute_implicit_vjp, solve_adjoint
from difffea_b200.newton_krylov import solve_newton_krylov


class EquilibriumSolve(torch.autograd.Function):
    @staticmethod
    def forward(ctx, theta, params, options):
        opts = dict(options)
        adj = {k: opts.pop(k) for k in ("adjoint_rtol", "adjoint_max_iter", "adjoint_preconditioner",
                                        "adjoint_on_failure") if k in opts}
        opts.setdefault("verbose", False)
        u = solve_newton_krylov(params, theta.detach(), **opts)
        ctx.save_for_backward(theta.detach(), u)
        ctx.params = params
        ctx.adjoint = adj
        return u

    @staticmethod
    def backward(ctx, grad_u):
        theta, u = ctx.saved_tensors
        lam, iters, status = solve_adjoint(u, theta, ctx.params, grad_u.contiguous(),
                                           rtol=ctx.adjoint.get("adjoint_rtol", 1e-10),
                                           max_iter=ctx.adjoint.get("adjoint_max_iter", 500),
                                           preconditioner=ctx.adjoint.get("adjoint_preconditioner", "auto"),
                                           on_failure=ctx.adjoint.get("adjoint_on_failure", "warn"),
                                           return_status=True)
        ctx.adjoint_iterations, ctx.adjoint_status = iters, status
        return compute_implicit_vjp(u, theta, ctx.params, lam).to(theta.dtype), None, None


def equilibrium(theta, params, **options):
    """u*(theta), differentiable w.r.t. theta through the adjoint."""
    return EquilibriumSolve.apply(theta, params, options)


def compliance(theta, params, **options):
    """L(theta) = f . u*(theta), differentiable w.r.t. theta."""
    return torch.dot(params["f"].to(torch.float64), equilibrium(theta, params, **options))
