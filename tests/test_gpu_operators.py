"""
Parity of kernels (a) and (b), the residual and the strain energy with the reference (golden vectors)
and the oracle, FP64 and FP32, plus determinism, symmetry and linearity at larger sizes.
"""
import pytest
import torch

import oracle
from difffea_b200 import ops
from difffea_b200.cuda_mesh import cuda_mesh
from difffea_b200.materials import device_material, neo_hookean_parameters
from difffea_b200.operators import global_residual, make_A_operator_cuda, make_tangent_operator, strain_energy
from difffea_b200.problem import build_rectangle_problem, to_device
from golden_utils import golden_names, load, params_from, rel

pytestmark = pytest.mark.gpu
DEV = "cuda"
OPERATOR_CASES = golden_names("operator_")


def unpack_moduli(mesh, C):
    """(n_el, n_q, 4, 4) in original element order from the colour-sorted SoA layout of kernel (a)."""
    S, nq, n = mesh.stride, mesh.n_q, mesh.n_el
    if C.dtype == torch.float64:
        slot = C.view(nq, 8, S, 2)[:, :, :n, :].permute(2, 0, 1, 3).reshape(n, nq, 4, 4)
    else:
        slot = C.view(nq, 4, S, 4)[:, :, :n, :].permute(2, 0, 1, 3).reshape(n, nq, 4, 4)
    out = torch.empty_like(slot)
    out[mesh.perm] = slot
    return out


def golden_case(name):
    d = load(name)
    p = params_from(d, DEV)
    t = lambda k: torch.as_tensor(d[k], dtype=torch.float64, device=DEV)  # noqa: E731
    return d, p, t("u"), t("v"), t("theta")


@pytest.mark.parametrize("name", OPERATOR_CASES)
def test_moduli_and_diagonal_match_reference(name):
    d, p, u, v, th = golden_case(name)
    A = make_A_operator_cuda(u, th, p)
    assert rel(unpack_moduli(A.mesh, A.C), d["C"]) < 1e-12
    assert rel(A.diag, d["diag"]) < 1e-12


@pytest.mark.parametrize("name", OPERATOR_CASES)
def test_tangent_product_matches_qp_ew(name):
    d, p, u, v, th = golden_case(name)
    y = make_tangent_operator("cuda", u, th, p)(v)
    assert rel(y, d["Av_qp_ew"]) < 1e-11           # the parity bar per product
    assert rel(y, d["Av_jvp"]) < 1e-11
    assert make_tangent_operator("auto", u, th, p)(v).equal(y)


@pytest.mark.parametrize("name", OPERATOR_CASES)
def test_residual_and_energy_match_reference(name):
    d, p, u, v, th = golden_case(name)
    assert rel(global_residual(u, th, p), d["R"]) < 1e-12
    assert rel(global_residual(u, th, p, load_factor=0.5), d["R_half"]) < 1e-12
    W = float(strain_energy(u, th, p))
    assert abs(W - float(d["energy"])) <= 1e-12 * abs(float(d["energy"]))


@pytest.mark.parametrize("name", OPERATOR_CASES)
def test_fp32_operator_is_close(name):
    d, p, u, v, th = golden_case(name)
    A32 = make_A_operator_cuda(u, th, p, precision="fp32")
    y = A32(v.float())
    assert y.dtype == torch.float32
    assert rel(y.double(), d["Av_qp_ew"]) < 2e-5
    assert rel(unpack_moduli(A32.mesh, A32.C).double(), d["C"]) < 1e-6


def _random_state(p, h, seed):
    g = torch.Generator(device="cpu").manual_seed(seed)
    n = p["f"].shape[0]
    u = ((torch.rand(n, dtype=torch.float64, generator=g) * 2 - 1) * 0.05 * h).to(DEV) * p["m"]
    v = torch.randn(n, dtype=torch.float64, generator=g).to(DEV)
    w = torch.randn(n, dtype=torch.float64, generator=g).to(DEV)
    th = torch.exp(0.3 * torch.randn(p["conn"].shape[0], dtype=torch.float64, generator=g)).to(DEV)
    return u, v, w, th


@pytest.mark.parametrize("et,nx,ny", [("quad4", 120, 60), ("quad9", 40, 20), ("tri6", 30, 20), ("tri3", 60, 30),
                                      ("quad8", 30, 15)])
def test_larger_meshes_against_oracle(et, nx, ny):
    p = build_rectangle_problem(et, nx, ny, float(nx), float(ny), load=(0.0, 1e-3), device=DEV)
    u, v, w, th = _random_state(p, 1.0, 7)
    P = oracle.as_problem(p)
    A = make_tangent_operator("cuda", u, th, p)
    uc, thc, vc = u.cpu(), th.cpu(), v.cpu()
    C_ref = oracle.moduli(uc, thc, P)
    assert rel(A(v), oracle.apply_qp_ew(C_ref, vc, P)) < 1e-11
    assert rel(global_residual(u, th, p, 0.7), oracle.residual(uc, thc, P, 0.7)) < 1e-12
    assert rel(A.diag, oracle.jacobi_diagonal(uc, thc, P)) < 1e-12


@pytest.mark.parametrize("et", ["quad4", "quad9"])
def test_product_is_deterministic_symmetric_and_linear(et):
    n = 160 if et == "quad4" else 80
    p = build_rectangle_problem(et, n, n, float(n), float(n), device=DEV)
    u, v, w, th = _random_state(p, 1.0, 3)
    A = make_tangent_operator("cuda", u, th, p)
    y1, y2 = A(v), A(v)
    assert torch.equal(y1, y2)                                       # colour-ordered scatter: bitwise
    Aw = A(w)
    assert abs(float(w @ y1) - float(v @ Aw)) <= 1e-12 * abs(float(v @ Aw))
    assert rel(A(2.5 * v - 0.5 * w), 2.5 * y1 - 0.5 * Aw) < 1e-13
    fixed = ~p["m"].bool()
    e = torch.zeros_like(v)
    e[fixed] = v[fixed]
    assert torch.equal(A(e), e)                                      # identity pivot on fixed DOFs


def test_inverted_element_propagates_nan_like_the_reference():
    p = build_rectangle_problem("quad4", 4, 4, 4.0, 4.0, device=DEV)
    u = torch.zeros(p["f"].shape[0], dtype=torch.float64, device=DEV)
    th = torch.ones(p["conn"].shape[0], dtype=torch.float64, device=DEV)
    node = int(p["conn"][5, 2])
    u[2 * node] = -3.0                                               # fold one element over itself
    R = global_residual(u, th, p)
    R_ref = oracle.residual(u.cpu(), th.cpu(), oracle.as_problem(p))
    assert torch.equal(torch.isnan(R).cpu(), torch.isnan(R_ref))
    assert torch.isnan(R).any()


def test_custom_ops_are_registered():
    for name in ("tangent_apply", "qp_moduli", "residual", "element_sensitivity", "element_fields", "node_fields",
                 "internal_force", "pcg_solve", "mg_setup", "mg_vcycle", "mg_pcg", "newton_solve", "residual_out",
                 "qp_moduli_out", "add_scaled_out"):
        assert hasattr(torch.ops.difffea_b200, name), name
    d, p, u, v, th = golden_case("operator_quad4_h0.5_unit")
    mesh = cuda_mesh(p)
    mid = ops.register_mesh(mesh)
    C, _ = torch.ops.difffea_b200.qp_moduli(mid, u, th, *ops.material_args(device_material(p)), False, False)
    assert rel(torch.ops.difffea_b200.tangent_apply(mid, C, v), d["Av_qp_ew"]) < 1e-11


def test_reference_built_dictionary_on_device_is_accepted():
    """A params dict moved with to_device (reference layout) runs unchanged."""
    d = load("operator_tri6_h0.5_unit")
    p = to_device(params_from(d), DEV)
    u = torch.as_tensor(d["u"], device=DEV)
    y = make_tangent_operator("cuda", u, torch.ones(p["conn"].shape[0], dtype=torch.float64, device=DEV), p)(
        torch.as_tensor(d["v"], device=DEV))
    assert rel(y, d["Av_qp_ew"]) < 1e-11


@pytest.mark.parametrize("name", ["operator_quad4_h0.1_theta", "operator_quad9_h0.25_theta"])
def test_fp32_moduli_on_fp64_vectors(name):
    """The mixed operator: FP32 moduli and gradients applied to FP64 vectors in FP64 arithmetic."""
    d, p, u, v, th = golden_case(name)
    A32 = make_A_operator_cuda(u, th, p, precision="fp32")
    y = A32(v)
    assert y.dtype == torch.float64
    assert rel(y, d["Av_qp_ew"]) < 2e-6


# ------------------------------------------------------------------------------------------------
# gather form of the product: one element pass + per-node sums in the incidence order
# ------------------------------------------------------------------------------------------------
def _apply_gather(A, v):
    from difffea_b200 import _lib
    from difffea_b200.cuda_mesh import ptr, stream_handle
    A.mesh.ensure_node_incidence()
    vcode = _lib.DFEA_F32 if v.dtype == torch.float32 else _lib.DFEA_F64
    fe = torch.empty(int(_lib.load().dfea_gather_work_bytes(A.mesh.view_ref, vcode)), dtype=torch.uint8, device=DEV)
    y = torch.empty_like(v)
    cdt = _lib.DFEA_F32 if A.C.dtype == torch.float32 else _lib.DFEA_F64
    _lib.call("dfea_tangent_apply_gather", A.mesh.view_ref, ptr(A.C), cdt, ptr(v), ptr(y), vcode, ptr(fe),
              stream_handle())
    return y


@pytest.mark.parametrize("name", OPERATOR_CASES)
def test_gather_form_product_matches_qp_ew(name):
    d, p, u, v, th = golden_case(name)
    A = make_tangent_operator("cuda", u, th, p)
    y = _apply_gather(A, v)
    assert rel(y, d["Av_qp_ew"]) < 1e-11
    assert rel(y, A(v)) < 1e-13                                     # same operator as the colour form
    assert torch.equal(y, _apply_gather(A, v))                      # fixed summation order: bitwise


@pytest.mark.parametrize("et,nx,ny", [("quad4", 160, 160), ("quad9", 60, 40), ("tri6", 40, 30)])
def test_gather_form_at_size_fp64_and_fp32(et, nx, ny):
    p = build_rectangle_problem(et, nx, ny, float(nx), float(ny), device=DEV)
    u, v, w, th = _random_state(p, 1.0, 9)
    A = make_tangent_operator("cuda", u, th, p)
    assert rel(_apply_gather(A, v), A(v)) < 1e-13
    A32 = make_A_operator_cuda(u, th, p, precision="fp32")
    assert rel(_apply_gather(A32, v.float()).double(), A32(v.float()).double()) < 1e-5
    assert rel(_apply_gather(A32, v), A32(v)) < 1e-13              # mixed: FP32 operator data, FP64 vectors


# ------------------------------------------------------------------------------------------------
# reference-frame FP32 moduli (DFEA_F32REF): 10 per Gauss point, no gradients read by the product
# ------------------------------------------------------------------------------------------------
def _ref_operator(p, u, th):
    from difffea_b200 import _lib
    from difffea_b200.cuda_mesh import ptr, stream_handle
    mesh = cuda_mesh(p)
    mesh.ensure_ref_frame()
    mesh.ensure_node_incidence()
    mu0, lam0 = neo_hookean_parameters(p)
    C = torch.empty(mesh.moduli_numel_ref(), dtype=torch.float32, device=DEV)
    _lib.call("dfea_qp_moduli", mesh.view_ref, ptr(u.contiguous()), ptr(th.contiguous()), mu0, lam0, ptr(C),
              _lib.DFEA_F32REF, ptr(None), stream_handle())
    return mesh, C


def _ref_apply(mesh, C, v, gather):
    from difffea_b200 import _lib
    from difffea_b200.cuda_mesh import ptr, stream_handle
    y = torch.empty_like(v)
    if gather:
        fe = torch.empty(int(_lib.load().dfea_gather_work_bytes(mesh.view_ref, _lib.DFEA_F64)), dtype=torch.uint8,
                         device=DEV)
        _lib.call("dfea_tangent_apply_gather", mesh.view_ref, ptr(C), _lib.DFEA_F32REF, ptr(v), ptr(y), _lib.DFEA_F64,
                  ptr(fe), stream_handle())
    else:
        _lib.call("dfea_tangent_apply", mesh.view_ref, ptr(C), _lib.DFEA_F32REF, ptr(v), ptr(y), _lib.DFEA_F64,
                  stream_handle())
    return y


@pytest.mark.parametrize("name", OPERATOR_CASES)
def test_reference_frame_fp32_operator_matches_qp_ew(name):
    d, p, u, v, th = golden_case(name)
    mesh, C = _ref_operator(p, u, th)
    y_col, y_gat = _ref_apply(mesh, C, v, False), _ref_apply(mesh, C, v, True)
    assert rel(y_col, d["Av_qp_ew"]) < 2e-6 and rel(y_gat, d["Av_qp_ew"]) < 2e-6
    assert rel(y_col, y_gat) < 1e-13                                  # same FP32 data, FP64 arithmetic
    assert torch.equal(y_gat, _ref_apply(mesh, C, v, True))


@pytest.mark.parametrize("et,nx,ny", [("quad4", 120, 60), ("quad9", 40, 20), ("tri6", 30, 20)])
def test_reference_frame_operator_at_size_is_symmetric(et, nx, ny):
    p = build_rectangle_problem(et, nx, ny, float(nx), float(ny), device=DEV)
    u, v, w, th = _random_state(p, 1.0, 5)
    mesh, C = _ref_operator(p, u, th)
    Av, Aw = _ref_apply(mesh, C, v, True), _ref_apply(mesh, C, w, True)
    assert abs(float(w @ Av) - float(v @ Aw)) <= 1e-10 * abs(float(v @ Aw))   # FP32 data, exact symmetry kept
    assert rel(Av, make_tangent_operator("cuda", u, th, p)(v)) < 2e-6


@pytest.mark.parametrize("case", ["quad4", "quad9", "quad8", "tri3", "tri6", "plate_quad9"])
def test_reference_frame_jacobians_match_the_node_geometry(case):
    """The library's packed inverse Jacobians equal (dX/dxi)^-1 formed from the nodes with torch (the mapped
    quarter plate: a different Jacobian in every element)."""
    from difffea_b200.problem import build_quarter_plate_problem
    p = (build_quarter_plate_problem("quad9", n_theta=6, n_radial=5, device=DEV) if case == "plate_quad9"
         else build_rectangle_problem(case, 7, 3, 2.0, 1.1, device=DEV))
    mesh = cuda_mesh(p)
    jinv = mesh.ensure_ref_frame()
    S, nq, nen, n = mesh.stride, mesh.n_q, mesh.nen, mesh.n_el
    conn = (mesh.conn.view(nen, S)[:, :n] >> 2).to(torch.int64).t()
    X = p["nodes"].to(torch.float64)[conn]                                   # (n, nen, 2), packed order
    J = torch.einsum("eai,qaj->eqij", X, mesh.ref_grad.to(X.device))
    det = J[..., 0, 0] * J[..., 1, 1] - J[..., 0, 1] * J[..., 1, 0]
    inv = torch.stack([torch.stack([J[..., 1, 1], -J[..., 0, 1]], -1),
                       torch.stack([-J[..., 1, 0], J[..., 0, 0]], -1)], -2) / det[..., None, None]
    expect = torch.zeros(nq, 2, S, 2, dtype=torch.float64, device=X.device)
    expect[:, :, :n, :] = inv.permute(1, 2, 0, 3)
    assert float((jinv - expect).abs().max()) <= 1e-14 * float(expect.abs().max())


@pytest.mark.parametrize("case", ["quad4", "quad9", "quad8", "tri6", "plate_quad9"])
def test_node_incidence_is_the_stable_sort_of_the_slots_by_node(case):
    """The library's node incidence (counting, scan, fill, per-node sort) equals the CSR a stable sort of the
    packed slots a * stride + e by node gives, bit for bit."""
    from difffea_b200.problem import build_quarter_plate_problem
    p = (build_quarter_plate_problem("quad9", n_theta=6, n_radial=5, device=DEV) if case == "plate_quad9"
         else build_rectangle_problem(case, 9, 4, 2.0, 1.1, device=DEV))
    mesh = cuda_mesh(p)
    ptr_, inc = mesh.ensure_node_incidence()
    S, nen, n, N = mesh.stride, mesh.nen, mesh.n_el, mesh.n_nodes
    nodes = (mesh.conn.view(nen, S)[:, :n] >> 2).to(torch.int64).reshape(-1)
    flat = (torch.arange(nen, device=nodes.device)[:, None] * S + torch.arange(n, device=nodes.device)[None, :]).reshape(-1)
    expect_inc = flat[torch.sort(nodes, stable=True).indices].to(torch.int32)
    expect_ptr = torch.zeros(N + 1, dtype=torch.int64, device=nodes.device)
    expect_ptr[1:] = torch.cumsum(torch.bincount(nodes, minlength=N), 0)
    assert torch.equal(inc, expect_inc) and torch.equal(ptr_, expect_ptr.to(torch.int32))


def test_reference_frame_rejects_inconsistent_geometry():
    d, p, u, v, th = golden_case("operator_quad4_h0.5_unit")
    q = dict(p)
    q["dN_dX"] = p["dN_dX"].flip(1).contiguous()                        # Gauss points in another order
    with pytest.raises(ValueError):
        cuda_mesh(q).ensure_ref_frame()


@pytest.mark.parametrize("name", OPERATOR_CASES)
def test_block_jacobi_matches_reference(name):
    from difffea_b200.operators import make_preconditioner
    d, p, u, v, th = golden_case(name)
    M = make_preconditioner("block_jacobi", u, th, p)
    assert rel(M(v), d["Minv_block_v"]) < 1e-12
