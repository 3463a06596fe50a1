"""
Pin the oracle (the CPU restatement used as the parity checker) to the reference's own outputs:
every golden vector in tests/golden was produced by the reference package (make_golden.py).
"""
import pytest
import torch

import oracle
from golden_utils import golden_names, load, params_from, rel

OPERATOR_CASES = golden_names("operator_")
SOLVE_CASES = golden_names("solve_")
SENS_CASES = golden_names("sensitivity_")
MAT_OPERATOR_CASES = [n for n in golden_names("material_") if not n.startswith(("material_solve", "material_sens"))]
MAT_SOLVE_CASES = golden_names("material_solve_")
MAT_SENS_CASES = golden_names("material_sensitivity_")


@pytest.mark.parametrize("name", OPERATOR_CASES)
def test_oracle_operator_quantities_match_reference(name):
    d = load(name)
    P = oracle.as_problem(params_from(d))
    u, v, th = (torch.as_tensor(d[k]) for k in ("u", "v", "theta"))
    C = oracle.moduli(u, th, P)
    assert rel(C, d["C"]) < 1e-13
    assert rel(oracle.apply_qp_ew(C, v, P), d["Av_qp_ew"]) < 1e-13
    assert rel(oracle.apply_qp(C, v, P), d["Av_qp"]) < 1e-13
    assert rel(oracle.make_operator("jvp", u, th, P)(v), d["Av_jvp"]) < 1e-12
    assert rel(oracle.residual(u, th, P), d["R"]) < 1e-13
    assert rel(oracle.residual(u, th, P, 0.5), d["R_half"]) < 1e-13
    assert rel(oracle.jacobi_diagonal(u, th, P), d["diag"]) < 1e-13
    assert rel(oracle.block_jacobi(u, th, P)(v), d["Minv_block_v"]) < 1e-12
    assert abs(float(oracle.strain_energy(u, th, P)) - float(d["energy"])) <= 1e-12 * abs(float(d["energy"]))


FIELD_KEYS = ("J", "sxx", "syy", "sxy", "mises", "energy_density", "ux", "uy", "u_mag", "strain_energy", "min_J",
              "ux_n", "uy_n", "u_mag_n", "J_n", "sxx_n", "syy_n", "sxy_n", "mises_n", "energy_density_n")


@pytest.mark.parametrize("name", OPERATOR_CASES + SOLVE_CASES)
def test_oracle_fields_and_reactions_match_reference(name):
    """compute_fields and support_reactions (postprocess.py:70-137) at the operator states and solutions."""
    d = load(name)
    P = oracle.as_problem(params_from(d))
    u = torch.as_tensor(d["u"] if "u" in d else d["u_star"])
    th = torch.as_tensor(d["theta"])
    out = oracle.compute_fields(u, th, P)
    assert sorted(out) == sorted(FIELD_KEYS)
    for k in FIELD_KEYS:
        assert rel(out[k], d["fields_" + k]) < 1e-12, k
    R = oracle.support_reactions(u, th, P)
    assert rel(R, d["reactions"]) < 1e-12
    if "u_star" in d:                 # equilibrium: reactions balance the applied load
        f = torch.as_tensor(d["f"]).reshape(-1, 2).sum(0)
        assert float((R + f).abs().max()) < 1e-6 * float(f.abs().max())


@pytest.mark.parametrize("name", SOLVE_CASES)
def test_oracle_solve_matches_reference(name):
    d = load(name)
    P = oracle.as_problem(params_from(d))
    th = torch.as_tensor(d["theta"])
    pre = str(d["preconditioner"]) if "preconditioner" in d else "jacobi"
    u, info = oracle.newton_krylov_solve(P, th, int(d["n_load_steps"]), float(d["tol"]), tangent="qp", precond=pre)
    assert info["converged"]
    assert rel(u, d["u_star"]) < 1e-9
    assert info["total_newton"] == int(d["total_newton"])
    assert abs(info["total_cg"] - int(d["total_cg"])) <= max(2, 0.02 * int(d["total_cg"]))


@pytest.mark.parametrize("name", SENS_CASES)
def test_oracle_sensitivity_matches_reference(name):
    d = load(name)
    P = oracle.as_problem(params_from(d))
    th = torch.as_tensor(d["theta"])
    u, g = oracle.compute_sensitivity(P, th, lambda w: torch.dot(P["f"], w), n_load_steps=2, tol=1e-12)
    assert rel(u, d["u_star"]) < 1e-9
    assert rel(g, d["dL_dtheta"]) < 1e-8


def test_dolfinx_known_answers():
    """Published dolfinx max |u| of the structured rectangle cases (benchmarks/results/validate_dolfinx.json)."""
    for name, known in (("solve_quad4_h0.25_cantilever", 0.5168860494403356),
                        ("solve_tri6_h0.5_cantilever", 0.5321248641215832)):
        d = load(name)
        assert abs(abs(d["u_star"]).max() - known) <= 1e-12 * known


def test_oracle_on_the_plate_fixture():
    """Quarter plate (mapped Q9): the reference's solution is an equilibrium of the oracle's residual."""
    d = load("plate_quad9_24x24")
    P = oracle.as_problem(params_from(d))
    u, th = torch.as_tensor(d["u_star"]), torch.as_tensor(d["theta"])
    assert float(torch.norm(oracle.residual(u, th, P))) < float(d["tol"])
    assert abs(float(oracle.strain_energy(u, th, P)) - float(d["energy"])) <= 1e-12 * abs(float(d["energy"]))


def test_oracle_on_the_gradient_fixture():
    """Log-normal cantilever: equilibrium, the adjoint equation and -lambda^T dR/dtheta of the oracle."""
    d = load("gradient_quad4_128x128")
    P = oracle.as_problem(params_from(d))
    u, th, lam = (torch.as_tensor(d[k]) for k in ("u_star", "theta", "lam"))
    assert float(torch.norm(oracle.residual(u, th, P))) < float(d["tol"])
    AT = oracle.make_transpose_operator(u, th, P)
    b = P["m"] * P["f"]
    assert float(torch.norm(AT(lam) - b)) <= 1.01e-10 * float(torch.norm(b))
    assert rel(oracle.implicit_vjp(u, th, P, lam), d["dL_dtheta"]) < 1e-12


# ---------------------------------------------------------------------------------------------
# the other materials of the library (materials.py:65-186)
# ---------------------------------------------------------------------------------------------
@pytest.mark.parametrize("name", MAT_OPERATOR_CASES)
def test_oracle_material_operator_quantities_match_reference(name):
    d = load(name)
    P = oracle.as_problem(params_from(d))
    u, v, th = (torch.as_tensor(d[k]) for k in ("u", "v", "theta"))
    C = oracle.moduli(u, th, P)
    assert rel(C, d["C"]) < 1e-12
    assert rel(oracle.apply_qp_ew(C, v, P), d["Av_qp_ew"]) < 1e-12
    assert rel(oracle.residual(u, th, P), d["R"]) < 1e-12
    assert rel(oracle.residual(u, th, P, 0.5), d["R_half"]) < 1e-12
    assert rel(oracle.jacobi_diagonal(u, th, P), d["diag"]) < 1e-12
    assert rel(oracle.block_jacobi(u, th, P)(v), d["Minv_block_v"]) < 1e-12
    assert abs(float(oracle.strain_energy(u, th, P)) - float(d["energy"])) <= 1e-12 * abs(float(d["energy"]))
    out = oracle.compute_fields(u, th, P)
    for k in FIELD_KEYS:
        assert rel(out[k], d["fields_" + k]) < 1e-12, k
    assert rel(oracle.support_reactions(u, th, P), d["reactions"]) < 1e-12


@pytest.mark.parametrize("name", MAT_SOLVE_CASES)
def test_oracle_material_solve_matches_reference(name):
    d = load(name)
    P = oracle.as_problem(params_from(d))
    th = torch.as_tensor(d["theta"])
    u, info = oracle.newton_krylov_solve(P, th, int(d["n_load_steps"]), float(d["tol"]), tangent="qp")
    assert info["converged"]
    assert rel(u, d["u_star"]) < 1e-9
    assert info["total_newton"] == int(d["total_newton"])


@pytest.mark.parametrize("name", MAT_SENS_CASES)
def test_oracle_material_sensitivity_matches_reference(name):
    d = load(name)
    P = oracle.as_problem(params_from(d))
    th = torch.as_tensor(d["theta"])
    f = P["f"]
    u, g = oracle.compute_sensitivity(P, th, lambda w: torch.dot(f, w), n_load_steps=2, tol=1e-12)
    assert rel(u, d["u_star"]) < 1e-9
    assert rel(g, d["dL_dtheta"]) < 1e-8
