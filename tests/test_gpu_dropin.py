"""
The drop-in, executed: the reference's own newton_krylov_solve (newton_krylov.py:185-264) with the "cuda"
tangent variant registered beside jvp / linearize / qp / qp_ew (difffea_b200.dropin.register applies the
lines a maintainer adds to operators.py:415-435 / 702-710 and newton_krylov.py:28).  The reference's Newton
loop, line search, continuation and residual run unchanged on CUDA tensors; the tangent operator, the
Jacobi (or multigrid) preconditioner and the PCG are this package's kernels.  The solution is compared with
the reference's own CUDA path (tangent "qp_ew") on the same problem, bar 1e-9.
"""
import pytest
import torch

import reference_package
from golden_utils import rel

pytestmark = pytest.mark.gpu
REF = reference_package.load()
needs_reference = pytest.mark.skipif(REF is None, reason=reference_package.MISSING)


def _reference_problem(element_type, h):
    from difffea.problem import build_problem, default_spec, to_device
    spec = default_spec("rectangle", element_type, h)
    spec.update(mesher="structured", load_value=(60.0, 0.0), E=2600.0, nu=0.3)
    return to_device(build_problem(spec), "cuda")


@needs_reference
@pytest.mark.parametrize("element_type,h,preconditioner", [("quad4", 0.05, "jacobi"), ("quad9", 0.1, "jacobi"),
                                                           ("quad4", 0.05, "multigrid")])
def test_reference_solver_runs_the_cuda_variant(element_type, h, preconditioner):
    from difffea import newton_krylov as nk
    from difffea_b200.dropin import register
    p = _reference_problem(element_type, h)
    th = torch.ones(p["conn"].shape[0], dtype=torch.float64, device="cuda")
    u_ref, info_ref = nk.newton_krylov_solve(p, th, n_load_steps=2, tol=1e-9, verbose=False, tangent="qp_ew")
    undo = register(REF)
    try:
        assert "cuda" in REF.operators.TANGENT_OPERATORS
        u, info = nk.newton_krylov_solve(p, th, n_load_steps=2, tol=1e-9, verbose=False, tangent="cuda",
                                         preconditioner=preconditioner)
    finally:
        undo()
    assert "cuda" not in REF.operators.TANGENT_OPERATORS               # the package is as it was
    err = rel(u, u_ref)
    print(f"\nreference newton_krylov_solve, {element_type} h={h}, {preconditioner}: tangent 'cuda' vs 'qp_ew' "
          f"{err:.2e}; Newton {info['total_newton']} ({info_ref['total_newton']}), CG {info['total_cg']} "
          f"({info_ref['total_cg']})")
    assert info["converged"] and info_ref["converged"]
    assert err <= 1e-9
    if preconditioner == "jacobi":
        assert info["total_newton"] == info_ref["total_newton"]


@needs_reference
def test_registered_operator_matches_the_reference_products():
    """Inside the patched package, make_tangent_operator("cuda") equals its qp_ew and jvp products."""
    from difffea import operators as ops
    from difffea_b200.dropin import register
    p = _reference_problem("quad4", 0.1)
    g = torch.Generator().manual_seed(3)
    n = p["f"].shape[0]
    u = ((torch.rand(n, dtype=torch.float64, generator=g) * 2 - 1) * 0.01).to("cuda") * p["m"]
    v = torch.randn(n, dtype=torch.float64, generator=g).to("cuda")
    th = torch.ones(p["conn"].shape[0], dtype=torch.float64, device="cuda")
    undo = register(REF)
    try:
        y = ops.make_tangent_operator("cuda", u, th, p)(v)
        y_ew = ops.make_tangent_operator("qp_ew", u, th, p)(v)
        y_jvp = ops.make_tangent_operator("jvp", u, th, p)(v)
        d = ops.make_preconditioner("jacobi", u, th, p)
    finally:
        undo()
    assert rel(y, y_ew) < 1e-11 and rel(y, y_jvp) < 1e-11
    assert rel(d.diag, ops.compute_jacobi_diagonal(u, th, p)) < 1e-12
