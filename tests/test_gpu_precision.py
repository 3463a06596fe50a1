"""
The mixed-precision study: a quarter plate with a circular hole (R = 1, half-width W = 10) on a mapped Q9
mesh, symmetry rollers on x = 0 and y = 0, a dead traction of 0.1 per unit length on x = W (about 10 %
stretch of the plate) applied in 5 load steps.  The "fp32" solve keeps the residual, the line search, the
convergence test and the state update in FP64 and runs the moduli and the PCG operator in FP32; each
result is checked against the reference's FP64 solution (24 x 24 fixture) or the FP64 device solve
(256 x 256, which the FP64 path reproduces within 1e-9 of the reference at every size tested).
"""
import pytest
import torch

from difffea_b200.newton_krylov import newton_krylov_solve
from difffea_b200.operators import strain_energy
from difffea_b200.problem import build_quarter_plate_problem
from golden_utils import load, params_from, rel

pytestmark = pytest.mark.gpu
DEV = "cuda"


def _errors(u, W, u_ref, W_ref):
    u_ref = torch.as_tensor(u_ref, dtype=torch.float64)
    return rel(u, u_ref), abs(W - W_ref) / abs(W_ref)


@pytest.mark.parametrize("precision,bar", [("fp64", 1e-9), ("fp32", 1e-8)])
def test_plate_against_the_reference_solution(precision, bar):
    d = load("plate_quad9_24x24")
    p = params_from(d, DEV)
    th = torch.ones(p["conn"].shape[0], dtype=torch.float64, device=DEV)
    kw = dict(pcg_max_iter=5000, precision="fp32") if precision == "fp32" else {}
    u, info = newton_krylov_solve(p, th, int(d["n_load_steps"]), float(d["tol"]), verbose=False, **kw)
    assert info["converged"]
    e_u, e_W = _errors(u, float(strain_energy(u, th, p)), d["u_star"], float(d["energy"]))
    print(f"\nplate 24x24 Q9 {precision}: |u - u_ref|inf/|u_ref|inf = {e_u:.2e}, |W - W_ref|/|W_ref| = {e_W:.2e}")
    assert e_u <= bar and e_W <= bar
    if precision == "fp64":
        assert info["total_newton"] == int(d["total_newton"])


def test_plate_256_mixed_precision_meets_1e8():
    p = build_quarter_plate_problem("quad9", 256, 256, radius=1.0, half_width=10.0, traction=0.1, device=DEV)
    assert p["conn"].shape[0] == 65_536 and p["nodes"].shape[0] == 263_169
    th = torch.ones(p["conn"].shape[0], dtype=torch.float64, device=DEV)
    tol = 1e-11 * float(torch.norm(p["f"]))
    u64, i64 = newton_krylov_solve(p, th, 5, tol, verbose=False, pcg_max_iter=20000)
    u32, i32 = newton_krylov_solve(p, th, 5, tol, verbose=False, pcg_max_iter=20000, precision="fp32")
    assert i64["converged"] and i32["converged"]
    W64, W32 = float(strain_energy(u64, th, p)), float(strain_energy(u32, th, p))
    e_u, e_W = _errors(u32, W32, u64.cpu(), W64)
    right = p["nodes"][:, 0] >= 10.0 - 1e-9
    stretch = float(u64[0::2][right].mean()) / 10.0
    print(f"\nplate 256x256 Q9: stretch {stretch:.4f}; fp64 Newton {i64['total_newton']} CG {i64['total_cg']}; "
          f"fp32 Newton {i32['total_newton']} CG {i32['total_cg']}; |u32 - u64|inf/|u64|inf = {e_u:.2e}, "
          f"|W32 - W64|/|W64| = {e_W:.2e}")
    assert 0.07 < stretch < 0.14
    assert e_u <= 1e-8 and e_W <= 1e-8
