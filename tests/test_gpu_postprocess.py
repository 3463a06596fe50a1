"""
Post-processing on the GPU (compute_fields / support_reactions, postprocess.py:70-137) against the
reference's own outputs (the fields_* and reactions arrays of every operator and solve fixture) and
against the oracle on a 128 x 128 Q9 state.  FP64 throughout; the tolerance is 1e-12 relative to the
largest entry of each field (the kernel evaluates the Cauchy stress in closed form, the reference through
autodiff of the 3D energy, and the nodal averages sum in incidence order instead of conn order).
"""
import pytest
import torch

import oracle
from difffea_b200.newton_krylov import newton_krylov_solve
from difffea_b200.operators import strain_energy
from difffea_b200.postprocess import compute_fields, element_fields, support_reactions
from difffea_b200.problem import build_rectangle_problem
from golden_utils import golden_names, load, params_from, rel

pytestmark = pytest.mark.gpu
DEV = "cuda"
FIELD_KEYS = ("J", "sxx", "syy", "sxy", "mises", "energy_density", "ux", "uy", "u_mag", "strain_energy", "min_J",
              "ux_n", "uy_n", "u_mag_n", "J_n", "sxx_n", "syy_n", "sxy_n", "mises_n", "energy_density_n")


@pytest.mark.parametrize("name", golden_names("operator_") + golden_names("solve_"))
def test_fields_and_reactions_match_the_reference(name):
    d = load(name)
    p = params_from(d, DEV)
    u = torch.as_tensor(d["u"] if "u" in d else d["u_star"], device=DEV)
    th = torch.as_tensor(d["theta"], device=DEV)
    out = compute_fields(u, th, p)
    assert sorted(out) == sorted(FIELD_KEYS)
    for k in FIELD_KEYS:
        assert out[k].device.type == "cuda" and out[k].dtype == torch.float64
        assert out[k].shape == d["fields_" + k].shape, k
        assert rel(out[k], d["fields_" + k]) < 1e-12, k
    assert rel(support_reactions(u, th, p), d["reactions"]) < 1e-12


def test_fields_against_the_oracle_128_quad9():
    p = build_rectangle_problem("quad9", 128, 128, 1.0, 1.0, E=1.0, nu=0.3, load=(0.0, -0.01), device=DEV)
    n_el, n = p["conn"].shape[0], p["f"].numel()
    g = torch.Generator().manual_seed(5)
    x, y = p["nodes"][:, 0], p["nodes"][:, 1]
    smooth = torch.stack([0.05 * x * y, -0.08 * x * x], 1).reshape(-1)        # bending-like, no inversion
    u = (smooth + 0.01 / 128 * torch.randn(n, dtype=torch.float64, generator=g).to(DEV)) * p["m"]
    th = (0.5 + torch.rand(n_el, dtype=torch.float64, generator=g)).to(DEV)
    out = compute_fields(u, th, p)
    ref = oracle.compute_fields(u.cpu(), th.cpu(), oracle.as_problem(p))
    for k in FIELD_KEYS:
        assert rel(out[k], ref[k]) < 1e-12, k
    assert abs(float(out["strain_energy"]) - strain_energy(u, th, p)) <= 1e-12 * abs(float(out["strain_energy"]))
    el = element_fields(u, th, p)
    assert rel(el[0].sum(), 1.0) < 1e-12                                # areas add up to the unit square
    R = support_reactions(u, th, p)
    assert rel(R, oracle.support_reactions(u.cpu(), th.cpu(), oracle.as_problem(p))) < 1e-11


def test_reactions_balance_the_load_at_a_device_solution():
    p = build_rectangle_problem("quad4", 64, 32, 2.0, 1.0, E=1.0, nu=0.3, load=(0.0, -0.004), device=DEV)
    th = torch.ones(p["conn"].shape[0], dtype=torch.float64, device=DEV)
    tol = 1e-11 * float(torch.norm(p["f"]))
    u, info = newton_krylov_solve(p, th, 2, tol, verbose=False, pcg_max_iter=5000)
    assert info["converged"]
    R = support_reactions(u, th, p)
    f = p["f"].view(-1, 2).sum(0)
    assert float((R + f).abs().max()) < 1e-8 * float(f.abs().max())
    out = compute_fields(u, th, p)
    assert float(out["min_J"]) > 0.9 and float(out["mises"].max()) > 0.0
