"""
The differentiation study: a unit-square Q4 cantilever (clamped at x = 0, dead shear traction 0.0072 on
x = 1, about 5 % tip deflection) whose per-element stiffness scale is log-normal, theta = exp(0.3 z) with
z ~ N(0, 1) seeded.  Compliance L = f . u* and dL/dtheta from the adjoint kernels behind
torch.autograd.Function, against the reference's torch.func adjoint (128 x 128 fixture) and against
central finite differences (step 1e-6) on 20 seeded elements of the 1024 x 1024 mesh (1,048,576 elements).
"""
import pytest
import torch

from difffea_b200.autograd import compliance, equilibrium
from difffea_b200.newton_krylov import newton_at_load
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
    assert abs(float(L) - float(d["compliance"])) <= 1e-9 * abs(float(d["compliance"]))
    assert rel(th_g.grad, d["dL_dtheta"]) < 1e-8


def test_cantilever_1m_gradient_against_central_differences():
    n = 1024
    p = build_rectangle_problem("quad4", n, n, 1.0, 1.0, E=1.0, nu=0.3, load=(0.0, -SHEAR), device=DEV,
                                build_on_device=True)
    n_el = p["conn"].shape[0]
    assert n_el == 1_048_576
    th = _theta(n_el).requires_grad_(True)
    f = p["f"]
    tol = 1e-13 * float(torch.norm(f))
    ws = NewtonWorkspace(p)
    solve_kw = dict(n_load_steps=1, tol=tol, pcg_max_iter=20000, workspace=ws)
    u_star = equilibrium(th, p, adjoint_rtol=1e-12, adjoint_max_iter=100000, **solve_kw)
    L = torch.dot(f, u_star)
    L.backward()
    g = th.grad
    u_star = u_star.detach()
    with torch.no_grad():
        tip = float(u_star[1::2].abs().max())
        ids = torch.randperm(n_el, generator=torch.Generator().manual_seed(1))[:20].tolist()
        eps, fd = 1e-6, []
        for e in ids:
            dL = []
            for s in (1.0, -1.0):
                t = th.detach().clone()
                t[e] += s * eps
                u, ok, _ = newton_at_load(u_star, t, p, 1.0, tol, 25, False, None, 0, pcg_max_iter=20000,
                                          workspace=ws)
                assert ok
                dL.append(float(torch.dot(f, u - u_star)))              # L(theta') - L(theta), no cancellation
            fd.append((dL[0] - dL[1]) / (2 * eps))
    fd = torch.tensor(fd, dtype=torch.float64)
    ga = g[ids].cpu()
    err = float(torch.norm(ga - fd) / torch.norm(fd))
    print(f"\ncantilever 1024x1024 Q4: L = {float(L):.6e}, tip deflection {tip:.4f}; "
          f"FD on 20 elements: |g - g_fd| / |g_fd| = {err:.2e}; max |g| on them {float(ga.abs().max()):.3e}")
    assert 0.03 < tip < 0.08
    assert err < 1e-3
