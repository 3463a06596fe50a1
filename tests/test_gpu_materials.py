"""
The other materials of the reference's library on the GPU (Mooney-Rivlin, Saint Venant-Kirchhoff, Demiray,
fibre-reinforced HGO; materials.py:65-186), against the reference's own outputs: moduli, tangent products,
residuals, Jacobi and block-Jacobi preconditioners, energies, post-processing fields and reactions on three
element types; complete Newton-Krylov solves; adjoint sensitivities (also with theta scaling only some
parameters).  The kernels differentiate each energy in forward mode on the device; tolerances as for the
neo-Hookean path: moduli, residuals and diagonals 1e-12, products 1e-11, solutions 1e-9, sensitivities 1e-8.
"""
import pytest
import torch

from difffea_b200 import _lib, ops
from difffea_b200.cuda_mesh import cuda_mesh, ptr, stream_handle
from difffea_b200.materials import device_material, material_vector
from difffea_b200.newton_krylov import newton_krylov_solve
from difffea_b200.operators import (compute_jacobi_diagonal, global_residual, make_A_operator_cuda,
                                    make_block_jacobi_preconditioner, make_tangent_operator, strain_energy)
from difffea_b200.postprocess import compute_fields, support_reactions
from difffea_b200.problem import build_rectangle_problem
from difffea_b200.sensitivity import compute_sensitivity
from golden_utils import golden_names, load, params_from, rel
from test_gpu_operators import unpack_moduli

pytestmark = pytest.mark.gpu
DEV = "cuda"
OPERATOR_CASES = [n for n in golden_names("material_") if not n.startswith(("material_solve", "material_sens"))]
SOLVE_CASES = golden_names("material_solve_")
SENS_CASES = golden_names("material_sensitivity_")
FIELD_KEYS = ("J", "sxx", "syy", "sxy", "mises", "energy_density", "ux", "uy", "u_mag", "strain_energy", "min_J",
              "ux_n", "uy_n", "u_mag_n", "J_n", "sxx_n", "syy_n", "sxy_n", "mises_n", "energy_density_n")


def _case(name):
    d = load(name)
    p = params_from(d, DEV)
    t = lambda k: torch.as_tensor(d[k], dtype=torch.float64, device=DEV)  # noqa: E731
    return d, p, t("u"), t("v"), t("theta")


@pytest.mark.parametrize("name", OPERATOR_CASES)
def test_material_operators_match_reference(name):
    d, p, u, v, th = _case(name)
    A = make_A_operator_cuda(u, th, p)
    assert rel(unpack_moduli(A.mesh, A.C), d["C"]) < 1e-12
    assert rel(A.diag, d["diag"]) < 1e-12
    assert rel(make_tangent_operator("cuda", u, th, p)(v), d["Av_qp_ew"]) < 1e-11
    assert rel(compute_jacobi_diagonal(u, th, p), d["diag"]) < 1e-12
    assert rel(make_block_jacobi_preconditioner(u, th, p)(v), d["Minv_block_v"]) < 1e-11
    assert rel(global_residual(u, th, p), d["R"]) < 1e-12
    assert rel(global_residual(u, th, p, 0.5), d["R_half"]) < 1e-12
    W = strain_energy(u, th, p)
    assert abs(W - float(d["energy"])) <= 1e-12 * abs(float(d["energy"]))


@pytest.mark.parametrize("name", OPERATOR_CASES)
def test_material_fields_and_reactions_match_reference(name):
    d, p, u, v, th = _case(name)
    out = compute_fields(u, th, p)
    for k in FIELD_KEYS:
        assert rel(out[k], d["fields_" + k]) < 1e-12, k
    assert rel(support_reactions(u, th, p), d["reactions"]) < 1e-12


@pytest.mark.parametrize("name", [n for n in OPERATOR_CASES if "_quad4_" in n and "partial" not in n])
def test_material_fp32_moduli(name):
    """FP32 moduli (physical and reference-frame) of the differentiated energies, applied to FP64 vectors."""
    d, p, u, v, th = _case(name)
    y64 = make_tangent_operator("cuda", u, th, p)(v)
    A32 = make_A_operator_cuda(u, th, p, precision="fp32")
    assert rel(A32(v), y64) < 2e-6
    mesh = cuda_mesh(p)
    mesh.ensure_ref_frame()
    C = torch.empty(mesh.moduli_numel_ref(), dtype=torch.float32, device=DEV)
    _lib.call("dfea_qp_moduli_mat", mesh.view_ref, ptr(u), ptr(th), device_material(p), ptr(C), _lib.DFEA_F32REF,
              ptr(None), ptr(None), stream_handle())
    y = torch.empty_like(v)
    _lib.call("dfea_tangent_apply", mesh.view_ref, ptr(C), _lib.DFEA_F32REF, ptr(v), ptr(y), _lib.DFEA_F64,
              stream_handle())
    assert rel(y, y64) < 2e-6


@pytest.mark.parametrize("name", SOLVE_CASES)
def test_material_solve_matches_reference(name):
    d = load(name)
    p = params_from(d, DEV)
    th = torch.as_tensor(d["theta"], device=DEV)
    u, info = newton_krylov_solve(p, th, int(d["n_load_steps"]), float(d["tol"]), verbose=False)
    assert info["converged"]
    assert rel(u, d["u_star"]) < 1e-9
    assert info["total_newton"] == int(d["total_newton"])
    f = p["f"].view(-1, 2).sum(0)
    assert float((support_reactions(u, th, p) + f).abs().max()) < 1e-6 * float(f.abs().max())


@pytest.mark.parametrize("name", SENS_CASES)
def test_material_sensitivity_matches_reference(name):
    d = load(name)
    p = params_from(d, DEV)
    th = torch.as_tensor(d["theta"], device=DEV)
    u, g = compute_sensitivity(p, th, lambda w: torch.dot(p["f"], w), n_load_steps=2, tol=1e-12)
    assert rel(u, d["u_star"]) < 1e-9
    assert rel(g, d["dL_dtheta"]) < 1e-8


def test_mixed_precision_solve_with_a_differentiated_material():
    """FP32 reference-frame moduli inside the FP64 Newton loop, Mooney-Rivlin 64 x 16 Q9: 1e-8 of FP64."""
    p = build_rectangle_problem("quad9", 64, 16, 4.0, 1.0, load=(0.0, -0.5), device=DEV, material="mooney_rivlin",
                                material_params={"c10": 40.0, "c01": 10.0, "kappa": 150.0})
    th = torch.ones(p["conn"].shape[0], dtype=torch.float64, device=DEV)
    tol = 1e-11 * float(torch.norm(p["f"]))
    u64, i64 = newton_krylov_solve(p, th, 3, tol, verbose=False, pcg_max_iter=5000)
    u32, i32 = newton_krylov_solve(p, th, 3, tol, verbose=False, pcg_max_iter=5000, precision="fp32")
    assert i64["converged"] and i32["converged"]
    assert rel(u32, u64) < 1e-8
    assert 0.05 < float(u64[1::2].abs().max()) < 2.0


def test_theta_on_a_nonlinear_parameter_is_rejected():
    """Demiray with theta scaling gamma: the sensitivity kernel refuses (the force is not linear in theta)."""
    d, p, u, v, th = _case("material_demiray_quad4_h0.25")
    p = dict(p, mat_scalable=torch.tensor([True, True, True], device=DEV))
    mesh = cuda_mesh(p)
    mid = ops.register_mesh(mesh)
    with pytest.raises(RuntimeError, match="nonlinearly"):
        ops.element_sensitivity(mid, u, v, *ops.material_args(device_material(p)))


def test_bad_material_is_rejected():
    d, p, u, v, th = _case("material_saint_venant_quad4_h0.25")
    mat = device_material(p)
    mat.model = 9
    mesh = cuda_mesh(p)
    R = torch.empty_like(u)
    rc = _lib.load().dfea_internal_force_mat(mesh.view_ref, ptr(u), ptr(th), mat, ptr(R), stream_handle())
    assert rc == 2 and "not built" in _lib.last_error()
    mat = device_material(p)
    mat.scalable = 0x4                                   # a third parameter that Saint Venant-Kirchhoff lacks
    rc = _lib.load().dfea_internal_force_mat(mesh.view_ref, ptr(u), ptr(th), mat, ptr(R), stream_handle())
    assert rc == 1
    with pytest.raises(ValueError):
        material_vector("fiber_reinforced", {"k3": 1.0})
