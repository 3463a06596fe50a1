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
import torch

from difffea_b200 import ops
from difffea_b200.newton_krylov import pcg
from difffea_b200.operators import _f64c, _prepare, make_AT_operator, make_preconditioner


def solve_adjoint(u_star, theta, params, dL_du, rtol=1e-6, max_iter=500, preconditioner="jacobi"):
    """
    (lambda (2N,), PCG iterations) of A^T lambda = m * dL/du at the converged state u_star.  ``preconditioner``:
    "jacobi" (the reference's), "block_jacobi", or "multigrid" (structured meshes; the iteration count no
    longer grows with the mesh, which matters for the tight adjoint tolerances of sensitivities).
    """
    b = (params["m"] * dL_du).to(torch.float64).contiguous()
    if preconditioner == "multigrid":
        from difffea_b200 import _lib
        from difffea_b200.operators import make_A_operator_cuda, multigrid_for
        A = make_A_operator_cuda(u_star, theta, params)          # A^T = A: the tangent is symmetric
        mg = multigrid_for(A.mesh, params)
        mg.setup(A.C, _lib.DFEA_F64, A.diag)
        lam = torch.empty_like(b)
        iters, _ = mg.pcg(b, lam, rtol, max_iter)
        return lam, iters
    AT = make_AT_operator(u_star, theta, params)
    Minv = make_preconditioner(preconditioner, u_star, theta, params)
    return pcg(AT, b, Minv, rtol=rtol, max_iter=max_iter)


def compute_implicit_vjp(u_star, theta, params, lambda_adj):
    """dL/dtheta (n_el,) = -lambda^T dR/dtheta (theta enters linearly, so no theta dependence remains)."""
    mesh, mid, mat = _prepare(u_star, theta, params)
    return ops.element_sensitivity(mid, _f64c(u_star), _f64c(lambda_adj), *ops.material_args(mat))
