"""
The C++ Newton-Krylov driver (dfea_newton_solve, driver="native") against the Python driver of the same
package: the same control flow (newton_krylov.py:94-264) over the same kernels, so the two give the same
iterates bit for bit -- solution, Newton and CG counts, history -- across the preconditioners (Jacobi,
block-Jacobi, multigrid), both precisions, load continuation with cut-backs and prescribed displacements.
"""
import pytest
import torch

from difffea_b200.newton_krylov import newton_krylov_solve
from difffea_b200.problem import build_rectangle_problem
from difffea_b200.workspace import NewtonWorkspace
from golden_utils import load, params_from, rel

pytestmark = pytest.mark.gpu
DEV = "cuda"


def _both(p, th, n_steps, tol, precision="fp64", preconditioner="jacobi", **kw):
    out = []
    for driver in ("python", "native"):
        ws = NewtonWorkspace(p, precision, preconditioner=preconditioner)
        out.append(newton_krylov_solve(p, th, n_steps, tol, verbose=False, workspace=ws, precision=precision,
                                       preconditioner=preconditioner, driver=driver, **kw))
    return out


def _same(a, b):
    (u0, i0), (u1, i1) = a, b
    assert torch.equal(u0, u1)
    for k in ("converged", "load_factor", "total_newton", "total_cg", "n_cutbacks"):
        assert i0[k] == i1[k], k
    assert [(r["step"], r["iteration"], r["cg_iters"], r["alpha"], r["residual"]) for r in i0["history"]] == \
           [(r["step"], r["iteration"], r["cg_iters"], r["alpha"], r["residual"]) for r in i1["history"]]


@pytest.mark.parametrize("name", ["solve_quad4_h0.25_cantilever", "solve_quad9_h0.5_cantilever",
                                  "solve_tri6_h0.5_cantilever", "solve_quad4_h0.2_tension_bj"])
def test_native_driver_reproduces_the_python_driver_on_reference_fixtures(name):
    d = load(name)
    p = params_from(d, DEV)
    th = torch.as_tensor(d["theta"], dtype=torch.float64, device=DEV)
    pre = str(d["preconditioner"]) if "preconditioner" in d else "jacobi"
    a, b = _both(p, th, int(d["n_load_steps"]), float(d["tol"]), preconditioner=pre)
    _same(a, b)
    assert rel(b[0], d["u_star"]) < 1e-9 and b[1]["total_newton"] == int(d["total_newton"])


@pytest.mark.parametrize("et,precision,preconditioner", [("quad4", "fp64", "multigrid"), ("quad9", "fp32", "multigrid"),
                                                         ("quad4", "fp32", "jacobi")])
def test_native_driver_on_cantilevers(et, precision, preconditioner):
    p = build_rectangle_problem(et, 48, 12, 4.0, 1.0, E=1.3, nu=0.33, load=(0.03, 0.0), device=DEV)
    th = torch.ones(p["conn"].shape[0], dtype=torch.float64, device=DEV)
    tol = 1e-10 * float(torch.norm(p["f"]))
    _same(*_both(p, th, 1, tol, precision=precision, preconditioner=preconditioner, pcg_max_iter=5000))


def test_native_driver_cutbacks_and_prescribed_displacements():
    # a displacement-controlled stretch of 50 % in one load step with at most 8 Newton iterations per level:
    # the continuation cuts the increment back several times before it converges (the oracle needs 5)
    p = build_rectangle_problem("quad4", 16, 8, 2.0, 1.0, load=(1.0, None), load_mode="displacement", device=DEV)
    th = torch.ones(p["conn"].shape[0], dtype=torch.float64, device=DEV)
    a, b = _both(p, th, 1, 1e-9, max_newton=8)
    _same(a, b)
    assert b[1]["converged"] and b[1]["n_cutbacks"] >= 1
    right = p["fixed"] & (p["u_D"] != 0)
    assert torch.allclose(b[0][right], p["u_D"][right])            # the prescribed displacements hold
