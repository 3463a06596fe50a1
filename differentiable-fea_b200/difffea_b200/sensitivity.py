"""compute_sensitivity (the reference's sensitivity.py:7-38): forward solve, dL/du, adjoint, implicit VJP."""
from torch.func import grad

from difffea_b200.adjoint import compute_implicit_vjp, solve_adjoint
from difffea_b200.newton_krylov import solve_newton_krylov


def compute_sensitivity(params, theta, loss_fn, n_load_steps=5, tol=1e-8, max_newton=25, adjoint_rtol=1e-10,
                        adjoint_max_iter=500, adjoint_preconditioner="jacobi", adjoint_on_failure="warn", **solver_kw):
    """
    (u_star, dL/dtheta) for a scalar loss L(u*): u* by the device Newton-Krylov solver, dL/du by
    autodiff of ``loss_fn``, the adjoint by the device PCG, dL/dtheta by the sensitivity kernel.
    ``solver_kw`` passes pcg_max_iter / precision / workspace to the forward solve.  An adjoint that stops
    short of ``adjoint_rtol`` is reported as ``solve_adjoint`` does (``adjoint_on_failure``).
    """
    theta = theta.detach()
    u_star = solve_newton_krylov(params, theta, n_load_steps=n_load_steps, tol=tol, max_newton=max_newton,
                                 verbose=False, **solver_kw)
    dL_du = grad(loss_fn)(u_star)
    lam, _ = solve_adjoint(u_star, theta, params, dL_du, rtol=adjoint_rtol, max_iter=adjoint_max_iter,
                           preconditioner=adjoint_preconditioner, on_failure=adjoint_on_failure)
    return u_star, compute_implicit_vjp(u_star, theta, params, lam)
