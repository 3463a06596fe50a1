"""Kernel (d) and the adjoint path: sensitivities against the reference, the oracle and finite differences."""
import pytest
import torch

import oracle
from difffea_b200.adjoint import compute_implicit_vjp, solve_adjoint
from difffea_b200.autograd import compliance
from difffea_b200.newton_krylov import solve_newton_krylov
from difffea_b200.sensitivity import compute_sensitivity
from golden_utils import golden_names, load, params_from, rel

pytestmark = pytest.mark.gpu
DEV = "cuda"


def _t(d, k):
    return torch.as_tensor(d[k], dtype=torch.float64, device=DEV)


@pytest.mark.parametrize("name", golden_names("sensitivity_"))
def test_sensitivity_matches_reference(name):
    d = load(name)
    p = params_from(d, DEV)
    f = p["f"]
    u, g = compute_sensitivity(p, _t(d, "theta"), lambda w: torch.dot(f, w), n_load_steps=2, tol=1e-12)
    assert rel(u, d["u_star"]) < 1e-9
    assert rel(g, d["dL_dtheta"]) < 1e-8


def test_sensitivity_kernel_matches_oracle_vjp():
    d = load("operator_quad9_h0.25_theta")
    p = params_from(d, DEV)
    u, th = _t(d, "u"), _t(d, "theta")
    lam = torch.randn(u.numel(), dtype=torch.float64, generator=torch.Generator().manual_seed(5)).to(DEV)
    g = compute_implicit_vjp(u, th, p, lam)
    g_ref = oracle.implicit_vjp(u.cpu(), th.cpu(), oracle.as_problem(p), lam.cpu())
    assert rel(g, g_ref) < 1e-12


def test_adjoint_solution_matches_oracle():
    d = load("solve_quad4_h0.2_tension")
    p = params_from(d, DEV)
    th = _t(d, "theta")
    u = _t(d, "u_star")
    lam, k = solve_adjoint(u, th, p, p["f"], rtol=1e-10, max_iter=2000)
    lam_ref, k_ref = oracle.solve_adjoint(u.cpu(), th.cpu(), oracle.as_problem(p), p["f"].cpu(), rtol=1e-10,
                                          max_iter=2000)
    assert abs(k - k_ref) <= 1 and rel(lam, lam_ref) < 1e-8


def test_autograd_function_gives_the_adjoint_gradient():
    d = load("sensitivity_quad4_h0.25")
    p = params_from(d, DEV)
    th = _t(d, "theta").requires_grad_(True)
    L = compliance(th, p, n_load_steps=2, tol=1e-12)
    L.backward()
    assert rel(th.grad, d["dL_dtheta"]) < 1e-8


def test_adjoint_gradient_matches_central_differences():
    d = load("sensitivity_quad4_h0.25")
    p = params_from(d, DEV)
    th = _t(d, "theta")
    f = p["f"]
    _, g = compute_sensitivity(p, th, lambda w: torch.dot(f, w), n_load_steps=2, tol=1e-12)
    eps, g_fd = 1e-6, torch.zeros_like(th)
    for i in range(th.numel()):
        tp, tm = th.clone(), th.clone()
        tp[i] += eps
        tm[i] -= eps
        Lp = torch.dot(f, solve_newton_krylov(p, tp, 2, 1e-12, verbose=False))
        Lm = torch.dot(f, solve_newton_krylov(p, tm, 2, 1e-12, verbose=False))
        g_fd[i] = (Lp - Lm) / (2 * eps)
    assert float(torch.norm(g - g_fd) / torch.norm(g_fd)) < 1e-6


@pytest.mark.parametrize("preconditioner", ["jacobi", "multigrid"])
def test_unconverged_adjoint_is_reported(preconditioner):
    """An adjoint PCG stopped by its iteration cap warns (default) or raises; a converged one is silent."""
    from difffea_b200.adjoint import AdjointConvergenceWarning
    d = load("solve_quad4_h0.2_tension")
    p = params_from(d, DEV)
    th, u = _t(d, "theta"), _t(d, "u_star")
    with pytest.warns(AdjointConvergenceWarning, match="max_iter"):
        _, k, status = solve_adjoint(u, th, p, p["f"], rtol=1e-14, max_iter=2, preconditioner=preconditioner,
                                     return_status=True)
    assert (k, status) == (2, "max_iter")
    with pytest.raises(RuntimeError, match="did not reach"):
        solve_adjoint(u, th, p, p["f"], rtol=1e-14, max_iter=2, preconditioner=preconditioner, on_failure="raise")
    import warnings
    with warnings.catch_warnings():
        warnings.simplefilter("error", AdjointConvergenceWarning)
        _, _, status = solve_adjoint(u, th, p, p["f"], rtol=1e-10, max_iter=2000, preconditioner=preconditioner,
                                     return_status=True)
    assert status == "converged"


def test_autograd_backward_reports_an_unconverged_adjoint():
    from difffea_b200.adjoint import AdjointConvergenceWarning
    d = load("sensitivity_quad4_h0.25")
    p = params_from(d, DEV)
    th = _t(d, "theta").requires_grad_(True)
    L = compliance(th, p, n_load_steps=2, tol=1e-12, adjoint_max_iter=2, adjoint_preconditioner="jacobi")
    with pytest.warns(AdjointConvergenceWarning):
        L.backward()
    th.grad = None
    L = compliance(th, p, n_load_steps=2, tol=1e-12, adjoint_max_iter=2, adjoint_preconditioner="jacobi",
                   adjoint_on_failure="raise")
    with pytest.raises(RuntimeError, match="did not reach"):
        L.backward()
    # the default ("auto": multigrid on this structured mesh) converges and matches the reference
    th.grad = None
    L = compliance(th, p, n_load_steps=2, tol=1e-12)
    L.backward()
    assert rel(th.grad, d["dL_dtheta"]) < 1e-8
