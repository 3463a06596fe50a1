"""
The differentiation study: a unit-square Q4 cantilever (clamped at x = 0, dead shear traction 0.0072 on
x = 1, about 5 % tip deflection) whose per-element stiffness scale is log-normal, theta = exp(0.3 z) with
z ~ N(0, 1) seeded.  Compliance L = f . u* and dL/dtheta from the adjoint kernels behind
torch.autograd.Function, against the reference's torch.func adjoint (128 x 128 fixture) and against
central finite differences on 20 seeded elements: step 1e-6 on the 128 x 128 mesh, step 1e-3 on the
1024 x 1024 mesh (1,048,576 elements).
"""
import pytest
import torch

from difffea_b200.autograd import compliance, equilibrium
from difffea_b200.newton_krylov import newton_at_load
from difffea_b200.operators import residual_and_norm
from difffea_b200.problem import build_rectangle_problem
from difffea_b200.sensitivity import compute_sensitivity
from difffea_b200.workspace import NewtonWorkspace
from golden_utils import load, params_from, rel

pytestmark = pytest.mark.gpu
DEV = "cuda"
SHEAR = 0.0072


def _theta(n_el):
    z = torch.randn(n_el, dtype=torch.float64, generator=torch.Generator().manual_seed(0))
    return torch.exp(0.3 * z).to(DEV)


def test_gradient_matches_the_reference_torch_func_adjoint():
    d = load("gradient_quad4_128x128")
    p = params_from(d, DEV)
    th = torch.as_tensor(d["theta"], device=DEV)
    assert torch.equal(th.cpu(), _theta(th.numel()).cpu())
    f = p["f"]
    u, g = compute_sensitivity(p, th, lambda w: torch.dot(f, w), n_load_steps=1, tol=float(d["tol"]),
                               adjoint_max_iter=20000)
    assert rel(u, d["u_star"]) < 1e-9
    assert rel(g, d["dL_dtheta"]) < 1e-8
    th_g = th.clone().requires_grad_(True)
    L = compliance(th_g, p, n_load_steps=1, tol=float(d["tol"]), adjoint_max_iter=20000)
    L.backward()
    assert abs(float(L.detach()) - float(d["compliance"])) <= 1e-9 * abs(float(d["compliance"]))
    assert rel(th_g.grad, d["dL_dtheta"]) < 1e-8


def _central_differences(p, th, u_star, tol, ids, eps, ws):
    """(L(theta + eps e_i) - L(theta - eps e_i)) / 2 eps, each solve warm-started from u*."""
    f, out = p["f"], []
    for e in ids:
        dL = []
        for s in (1.0, -1.0):
            t = th.clone()
            t[e] += s * eps
            u, ok, _ = newton_at_load(u_star, t, p, 1.0, tol, 25, False, None, 0, pcg_max_iter=20000, workspace=ws)
            assert ok, f"finite-difference solve at element {e} ({s:+.0f} eps) did not converge"
            dL.append(float(torch.dot(f, u - u_star)))                  # L(theta') - L(theta), no cancellation
        out.append((dL[0] - dL[1]) / (2 * eps))
    return torch.tensor(out, dtype=torch.float64)


def test_gradient_against_central_differences_128():
    """
    128 x 128: central differences on 20 seeded elements.  With step 1e-6 (the reference's FD check) a
    difference of two compliances is ~1e-10 of L, near what the solves' residual floor (about 6e-12 ||f||
    at this size) resolves, so it agrees to a few percent only; with step 1e-3 it agrees to 1e-4.
    """
    d = load("gradient_quad4_128x128")
    p = params_from(d, DEV)
    th = torch.as_tensor(d["theta"], device=DEV)
    tol = float(d["tol"])
    ws = NewtonWorkspace(p)
    u, g = compute_sensitivity(p, th, lambda w: torch.dot(p["f"], w), n_load_steps=1, tol=tol,
                               adjoint_max_iter=20000, workspace=ws)
    ids = torch.randperm(th.numel(), generator=torch.Generator().manual_seed(1))[:20].tolist()
    errs = {}
    for eps in (1e-6, 1e-3):
        fd = _central_differences(p, th, u, tol, ids, eps, ws)
        errs[eps] = float(torch.norm(g[ids].cpu() - fd) / torch.norm(fd))
    print(f"\ncantilever 128x128 Q4: FD on 20 elements: |g - g_fd| / |g_fd| = {errs[1e-6]:.2e} (step 1e-6), "
          f"{errs[1e-3]:.2e} (step 1e-3)")
    assert errs[1e-6] < 5e-2 and errs[1e-3] < 1e-4


def test_cantilever_1m_gradient_against_central_differences():
    """
    1024 x 1024 (1,048,576 elements): compliance gradient by the adjoint vs central differences on 20
    seeded elements.  One element's share of the compliance is ~1e-6 here, so a step of 1e-6 moves L by
    ~1e-12 of itself -- below what an FP64 solve of this size resolves (its residual stalls near 2e-11
    ||f||, measured).  The differences use a step of 1e-3 (truncation error ~1e-6 relative).
    """
    n = 1024
    p = build_rectangle_problem("quad4", n, n, 1.0, 1.0, E=1.0, nu=0.3, load=(0.0, -SHEAR), device=DEV,
                                build_on_device=True)
    n_el = p["conn"].shape[0]
    assert n_el == 1_048_576
    th = _theta(n_el).requires_grad_(True)
    f = p["f"]
    tol = 1e-10 * float(torch.norm(f))
    ws = NewtonWorkspace(p)
    u_star = equilibrium(th, p, adjoint_rtol=1e-10, adjoint_max_iter=100000, n_load_steps=1, tol=tol,
                         pcg_max_iter=20000, workspace=ws)
    L = torch.dot(f, u_star)
    L.backward()
    g = th.grad
    u_star = u_star.detach()
    assert residual_and_norm(u_star, th.detach(), p)[1] < tol          # the forward solve converged
    tip = float(u_star[1::2].abs().max())
    ids = torch.randperm(n_el, generator=torch.Generator().manual_seed(1))[:20].tolist()
    with torch.no_grad():
        fd = _central_differences(p, th.detach(), u_star, tol, ids, 1e-3, ws)
    ga = g[ids].cpu()
    err = float(torch.norm(ga - fd) / torch.norm(fd))
    print(f"\ncantilever 1024x1024 Q4: L = {float(L):.6e}, tip deflection {tip:.4f}; "
          f"FD (step 1e-3) on 20 elements: |g - g_fd| / |g_fd| = {err:.2e}; max |g| {float(ga.abs().max()):.3e}")
    assert 0.03 < tip < 0.08
    assert err < 1e-3


def test_multigrid_adjoint_matches_the_reference_gradient():
    """The same gradient with the multigrid preconditioner in the forward solve and in the adjoint (functional
    and autograd forms), in a fraction of the Jacobi adjoint's iterations."""
    d = load("gradient_quad4_128x128")
    p = params_from(d, DEV)
    th = torch.as_tensor(d["theta"], device=DEV)
    f, tol = p["f"], float(d["tol"])
    u, g = compute_sensitivity(p, th, lambda w: torch.dot(f, w), n_load_steps=1, tol=tol, adjoint_max_iter=500,
                               adjoint_preconditioner="multigrid", preconditioner="multigrid")
    assert rel(u, d["u_star"]) < 1e-9
    assert rel(g, d["dL_dtheta"]) < 1e-8
    th_g = th.clone().requires_grad_(True)
    L = compliance(th_g, p, n_load_steps=1, tol=tol, adjoint_max_iter=500, adjoint_preconditioner="multigrid",
                   preconditioner="multigrid")
    L.backward()
    assert rel(th_g.grad, d["dL_dtheta"]) < 1e-8
    from difffea_b200.adjoint import solve_adjoint
    lam_m, it_m = solve_adjoint(u, th, p, f, rtol=1e-10, max_iter=500, preconditioner="multigrid")
    lam_j, it_j = solve_adjoint(u, th, p, f, rtol=1e-10, max_iter=20000)
    print(f"\nadjoint PCG iterations to 1e-10 at 128 x 128: multigrid {it_m}, Jacobi {it_j}")
    assert rel(lam_m, lam_j) < 1e-8 and it_m * 10 < it_j
