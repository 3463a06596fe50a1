"""
Adjoint sensitivities on the GPU (the reference's adjoint.py API).

    solve_adjoint(u_star, theta, params, dL_du, rtol=1e-6, max_iter=500)      adjoint.py:31-69
    compute_implicit_vjp(u_star, theta, params, lambda_adj)                     adjoint.py:75-106

The adjoint system A^T lambda = m * dL/du is solved by the device PCG with the stored-moduli operator
(the hyperelastic tangent is symmetric, so A^T = A).  The implicit VJP  dL/dtheta = -lambda^T dR/dtheta
is kernel (d): one thread per element evaluates f_e(u*; dp/dtheta) and contracts it with the masked
adjoint, which is exact because every energy of the library is linear in its theta-scaled parameters, so
R_int is linear in theta_e.
"""
import warnings

import torch

from difffea_b200 import ops
from difffea_b200.newton_krylov import pcg
from difffea_b200.operators import _f64c, _prepare, make_AT_operator, make_preconditioner

ADJOINT_PRECONDITIONERS = ("jacobi", "block_jacobi", "multigrid", "auto")


class AdjointConvergenceWarning(RuntimeWarning):
    """The adjoint PCG ended without reaching its tolerance (iteration cap or non-positive curvature)."""


def _adjoint_preconditioner(kind, params, mesh):
    """"auto": multigrid when the mesh's cells form a logical grid (the iteration count then stays flat
    with the mesh size), Jacobi otherwise."""
    if kind != "auto":
        return kind
    from difffea_b200.multigrid import structured_grid
    return "multigrid" if structured_grid(params["conn"].to(mesh.device), mesh.n_nodes) is not None else "jacobi"


def _report(status, iters, rtol, max_iter, on_failure):
    if status in ("converged", "zero_rhs"):
        return
    msg = (f"adjoint PCG did not reach rtol {rtol:g}: status '{status}' after {iters} of at most {max_iter} "
           "iterations; the sensitivity built on this adjoint is inaccurate (raise adjoint_max_iter or use "
           "preconditioner='multigrid')")
    if on_failure == "raise":
        raise RuntimeError(msg)
    if on_failure == "warn":
        warnings.warn(msg, AdjointConvergenceWarning, stacklevel=3)


def solve_adjoint(u_star, theta, params, dL_du, rtol=1e-6, max_iter=500, preconditioner="jacobi", *,
                  on_failure="warn", return_status=False):
    """
    (lambda (2N,), PCG iterations) of A^T lambda = m * dL/du at the converged state u_star.  ``preconditioner``:
    "jacobi" (the reference's), "block_jacobi", "multigrid" (structured meshes; the iteration count no
    longer grows with the mesh, which matters for the tight adjoint tolerances of sensitivities) or "auto"
    (multigrid on structured meshes, else Jacobi).

    The reference returns the iterate silently when PCG stops short (iteration cap or p.Ap <= 0); here that
    case is reported: ``on_failure`` "warn" (default, an ``AdjointConvergenceWarning``), "raise"
    (``RuntimeError``) or "ignore".  ``return_status=True`` appends the PCG status word ("converged",
    "max_iter", "negative_curvature", "zero_rhs") to the returned tuple.
    """
    if preconditioner not in ADJOINT_PRECONDITIONERS:
        raise ValueError(f"Unknown preconditioner '{preconditioner}'. Choose one of {ADJOINT_PRECONDITIONERS}.")
    if on_failure not in ("warn", "raise", "ignore"):
        raise ValueError("on_failure must be 'warn', 'raise' or 'ignore'")
    b = (params["m"] * dL_du).to(torch.float64).contiguous()
    mesh, _, _ = _prepare(u_star, theta, params)
    preconditioner = _adjoint_preconditioner(preconditioner, params, mesh)
    if preconditioner == "multigrid":
        from difffea_b200 import _lib
        from difffea_b200.operators import make_A_operator_cuda, multigrid_for
        A = make_A_operator_cuda(u_star, theta, params)          # A^T = A: the tangent is symmetric
        mg = multigrid_for(A.mesh, params)
        mg.setup(A.C, _lib.DFEA_F64, A.diag)
        lam = torch.empty_like(b)
        iters, status = mg.pcg(b, lam, rtol, max_iter)
    else:
        AT = make_AT_operator(u_star, theta, params)
        Minv = make_preconditioner(preconditioner, u_star, theta, params)
        lam, iters = pcg(AT, b, Minv, rtol=rtol, max_iter=max_iter)
        status = AT.last_status if AT.last_status is not None else (
            "max_iter" if iters >= max_iter else "converged")
    _report(status, iters, rtol, max_iter, on_failure)
    return (lam, iters, status) if return_status else (lam, iters)


def compute_implicit_vjp(u_star, theta, params, lambda_adj):
    """dL/dtheta (n_el,) = -lambda^T dR/dtheta (theta enters linearly, so no theta dependence remains)."""
    mesh, mid, mat = _prepare(u_star, theta, params)
    return ops.element_sensitivity(mid, _f64c(u_star), _f64c(lambda_adj), *ops.material_args(mat))
