"""
The run-time registration of the "cuda" variant in the reference package (difffea_b200.dropin), on the CPU:
the names it adds, that the reference's own names keep working for its variants, that an unknown name still
raises the reference's ValueError, and that undo restores the package.  No kernel runs here.
"""
import pytest
import torch

import reference_package

REF = reference_package.load()
pytestmark = pytest.mark.skipif(REF is None, reason=reference_package.MISSING)


def test_register_adds_the_variant_and_undo_restores_the_package():
    from difffea import newton_krylov as nk
    from difffea import operators as ops
    from difffea_b200.dropin import register
    before = (ops.make_tangent_operator, ops.make_preconditioner, nk.pcg, nk.make_tangent_operator,
              ops.TANGENT_OPERATORS, ops.PRECONDITIONERS)
    undo = register(REF)
    try:
        assert register(REF) is undo                                  # registering twice is a no-op
        assert ops.TANGENT_OPERATORS[-1] == "cuda" and "multigrid" in ops.PRECONDITIONERS
        assert nk.make_tangent_operator is ops.make_tangent_operator  # the Newton loop sees the new dispatch
        with pytest.raises(ValueError, match="Unknown tangent operator"):
            ops.make_tangent_operator("nope", torch.zeros(2), torch.ones(1), {})
    finally:
        undo()
    after = (ops.make_tangent_operator, ops.make_preconditioner, nk.pcg, nk.make_tangent_operator,
             ops.TANGENT_OPERATORS, ops.PRECONDITIONERS)
    assert after == before


def test_registered_package_still_runs_its_own_cpu_variants():
    """A solve with the reference's CPU "qp" variant and Jacobi is untouched by the registration."""
    from difffea import newton_krylov as nk
    from difffea.problem import build_problem, default_spec
    from difffea_b200.dropin import register
    spec = default_spec("rectangle", "quad4", 0.5)
    spec.update(mesher="structured", load_value=(60.0, 0.0), E=2600.0, nu=0.3)
    p = build_problem(spec)
    th = torch.ones(p["conn"].shape[0], dtype=torch.float64)
    u0, i0 = nk.newton_krylov_solve(p, th, n_load_steps=1, tol=1e-9, verbose=False, tangent="qp")
    undo = register(REF)
    try:
        u1, i1 = nk.newton_krylov_solve(p, th, n_load_steps=1, tol=1e-9, verbose=False, tangent="qp")
    finally:
        undo()
    assert torch.equal(u0, u1) and i0["total_cg"] == i1["total_cg"]
