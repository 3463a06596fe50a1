"""
Kernel (c) and the Newton-Krylov driver: complete solves against the reference's, the device PCG
against the oracle's PCG (same recurrences), its edge cases, and the mixed-precision solve.
"""
import pytest
import torch

import oracle
from difffea_b200.krylov import DevicePCG
from difffea_b200.newton_krylov import newton_krylov_solve, pcg
from difffea_b200.operators import (make_A_operator_cuda, make_jacobi_preconditioner, make_tangent_operator,
                                    strain_energy)
from difffea_b200.problem import build_rectangle_problem
from difffea_b200.workspace import NewtonWorkspace
from golden_utils import golden_names, load, params_from, rel

pytestmark = pytest.mark.gpu
DEV = "cuda"
SOLVE_CASES = golden_names("solve_")
# the fixtures of the reference's ILU-preconditioned solve pin the CPU oracle; the device has no ILU
DEVICE_PRECONDITIONER_CASES = [n for n in SOLVE_CASES if not n.endswith("_ilu")]


def _t(d, k):
    return torch.as_tensor(d[k], dtype=torch.float64, device=DEV)


@pytest.mark.parametrize("name", SOLVE_CASES)
def test_complete_solve_matches_reference(name):
    d = load(name)
    p = params_from(d, DEV)
    pre = str(d["preconditioner"]) if "preconditioner" in d else "jacobi"
    # the reference's ILU (a SciPy factorisation on the CPU) is not built on the device: its fixtures pin the
    # equilibrium, reached here with the multigrid-preconditioned device PCG (iteration counts then differ)
    device_pre = "multigrid" if pre == "ilu" else pre
    u, info = newton_krylov_solve(p, _t(d, "theta"), int(d["n_load_steps"]), float(d["tol"]), verbose=False,
                                  preconditioner=device_pre)
    assert info["converged"] and info["load_factor"] == 1.0
    assert rel(u, d["u_star"]) < 1e-9                      # the parity bar for complete solutions
    if device_pre == pre:
        assert info["total_newton"] == int(d["total_newton"])
        assert abs(info["total_cg"] - int(d["total_cg"])) <= max(3, 0.03 * int(d["total_cg"]))
    assert abs(float(strain_energy(u, _t(d, "theta"), p)) - float(d["energy"])) <= 1e-9 * abs(float(d["energy"]))


def test_dolfinx_known_answers_on_the_gpu():
    for name, known in (("solve_quad4_h0.25_cantilever", 0.5168860494403356),
                        ("solve_tri6_h0.5_cantilever", 0.5321248641215832)):
        d = load(name)
        p = params_from(d, DEV)
        u, info = newton_krylov_solve(p, _t(d, "theta"), 3, float(d["tol"]), verbose=False)
        assert abs(float(u.abs().max()) - known) <= 1e-10 * known


def _linear_system(name="operator_quad4_h0.1_theta"):
    d = load(name)
    p = params_from(d, DEV)
    u, th = _t(d, "u"), _t(d, "theta")
    P = oracle.as_problem(p)
    A = make_tangent_operator("cuda", u, th, p)
    M = make_jacobi_preconditioner(u, th, p)
    A_ref = oracle.make_operator("qp_ew", u.cpu(), th.cpu(), P)
    d_ref = oracle.jacobi_diagonal(u.cpu(), th.cpu(), P)
    b = p["m"] * _t(d, "v")
    return p, A, M, A_ref, d_ref, b


@pytest.mark.parametrize("rtol,max_iter", [(1e-10, 2000), (1e-4, 500), (1e-12, 5)])
def test_device_pcg_follows_the_reference_recurrences(rtol, max_iter):
    p, A, M, A_ref, d_ref, b = _linear_system()
    x, k = pcg(A, b, M, rtol=rtol, max_iter=max_iter)
    x_ref, k_ref = oracle.pcg(A_ref, b.cpu(), lambda r: r / d_ref, rtol=rtol, max_iter=max_iter)
    assert abs(k - k_ref) <= 1
    assert rel(x, x_ref) < (1e-9 if rtol < 1e-6 else 1e-6)


def test_device_pcg_zero_rhs_and_status():
    p, A, M, *_ = _linear_system()
    x, k = pcg(A, torch.zeros(A.mesh.n_dof, dtype=torch.float64, device=DEV), M)
    assert k == 0 and float(x.abs().max()) == 0.0 and A.last_status == "zero_rhs"


def test_device_pcg_negative_curvature_returns_z_at_first_iteration():
    d = load("operator_quad4_h0.25_theta")
    p = params_from(d, DEV)
    u, th = _t(d, "u"), -_t(d, "theta")                     # negated stiffness: p.Ap < 0 at once
    A = make_tangent_operator("cuda", u, th, p)
    M = make_jacobi_preconditioner(u, th, p)
    b = p["m"] * _t(d, "v")
    x, k = pcg(A, b, M)
    P = oracle.as_problem(p)
    x_ref, k_ref = oracle.pcg(oracle.make_operator("qp_ew", u.cpu(), th.cpu(), P), b.cpu(),
                              lambda r: r / oracle.jacobi_diagonal(u.cpu(), th.cpu(), P))
    assert k == k_ref == 0 and A.last_status == "negative_curvature"
    assert rel(x, x_ref) < 1e-12


def test_graph_and_direct_launch_give_identical_iterates():
    p, A, M, A_ref, d_ref, b = _linear_system()
    res = []
    for use_graph in (1, 2, 0):
        bb, xx = b.clone(), torch.empty_like(b)
        solver = DevicePCG(A.mesh, A.C, M.diag, bb, xx, use_graph=use_graph)
        k, status = solver.solve(1e-9, 1000)
        res.append((k, status, xx.clone()))
        solver.close()
    for k in (1, 2):
        assert res[0][0] == res[k][0] and res[0][1] == res[k][1] == "converged"
        assert torch.equal(res[0][2], res[k][2])


def test_mixed_precision_solve_meets_1e8():
    p = build_rectangle_problem("quad4", 40, 20, 2.0, 1.0, E=2600.0, load=(60.0, 0.0), device=DEV)
    th = torch.ones(p["conn"].shape[0], dtype=torch.float64, device=DEV)
    tol = 1e-12 * float(torch.norm(p["f"]))
    u64, i64 = newton_krylov_solve(p, th, 2, tol, verbose=False, pcg_max_iter=5000)
    u32, i32 = newton_krylov_solve(p, th, 2, tol, verbose=False, pcg_max_iter=5000, precision="fp32")
    assert i64["converged"] and i32["converged"]
    assert rel(u32, u64) <= 1e-8
    W64, W32 = float(strain_energy(u64, th, p)), float(strain_energy(u32, th, p))
    assert abs(W32 - W64) <= 1e-8 * abs(W64)


def test_load_cutbacks_recover():
    """One nominal step of a large tip load needs cut-backs (the continuation logic of the reference)."""
    p = build_rectangle_problem("quad4", 20, 4, 5.0, 1.0, E=1.0, load=(0.0, -0.08), device=DEV)
    th = torch.ones(p["conn"].shape[0], dtype=torch.float64, device=DEV)
    u, info = newton_krylov_solve(p, th, 1, 1e-9, max_newton=8, verbose=False, pcg_max_iter=2000)
    P = oracle.as_problem(p)
    u_ref, info_ref = oracle.newton_krylov_solve(P, th.cpu(), 1, 1e-9, max_newton=8, pcg_max_iter=2000)
    assert info["converged"] == info_ref["converged"]
    assert info["n_cutbacks"] == info_ref["n_cutbacks"]
    if info["converged"]:
        assert rel(u, u_ref) < 1e-7


# ------------------------------------------------------------------------------------------------
# gather form of the product inside the PCG iteration
# ------------------------------------------------------------------------------------------------
def _pcg_forms(A, b, rtol, max_iter, use_graph=1):
    out = {}
    for form in ("colour", "gather", "fused"):
        bb, xx = b.clone(), torch.empty_like(b)
        solver = DevicePCG(A.mesh, A.C, A.diag.to(b.dtype), bb, xx, use_graph=use_graph, form=form)
        k, status = solver.solve(rtol, max_iter)
        out[form] = (k, status, xx.clone())
        solver.close()
    return out


@pytest.mark.parametrize("name", ["operator_quad4_h0.1_theta", "operator_quad9_h0.25_theta",
                                  "operator_tri6_h0.25_theta", "operator_tri3_h0.25_theta",
                                  "operator_quad8_h0.25_theta"])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_gather_form_pcg_matches_the_colour_form(name, precision):
    d = load(name)
    p = params_from(d, DEV)
    u, th = 0.25 * _t(d, "u"), _t(d, "theta")                  # a milder state: SPD tangent for every type
    A = make_A_operator_cuda(u, th, p, precision=precision)
    b = p["m"] * _t(d, "v")                                     # FP64 vectors (mixed form for fp32 moduli)
    res = _pcg_forms(A, b, 1e-9, 3000)
    kc, sc, xc = res["colour"]
    for form in ("gather", "fused"):
        kg, sg, xg = res[form]
        assert sc == sg == "converged" and abs(kc - kg) <= 1
        assert rel(xg, xc) < 1e-8


@pytest.mark.parametrize("use_graph", [0, 1, 2])
@pytest.mark.parametrize("form", ["gather", "fused"])
def test_gather_form_is_reproducible_in_every_launch_form(use_graph, form):
    p, A, M, A_ref, d_ref, b = _linear_system()
    x_ref, k_ref = oracle.pcg(A_ref, b.cpu(), lambda r: r / d_ref, rtol=1e-10, max_iter=2000)
    runs = [_pcg_forms(A, b, 1e-10, 2000, use_graph)[form] for _ in range(2)]
    assert runs[0][:2] == runs[1][:2] and torch.equal(runs[0][2], runs[1][2])
    k, status, x = runs[0]
    assert status == "converged" and abs(k - k_ref) <= 1 and rel(x, x_ref) < 1e-9


def test_gather_form_zero_rhs_negative_curvature_and_cap():
    p, A, M, *_ = _linear_system()
    z = torch.zeros(A.mesh.n_dof, dtype=torch.float64, device=DEV)
    zr = _pcg_forms(A, z, 1e-9, 100)
    assert zr["gather"][:2] == zr["fused"][:2] == (0, "zero_rhs")
    d = load("operator_quad4_h0.25_theta")
    p = params_from(d, DEV)
    An = make_tangent_operator("cuda", _t(d, "u"), -_t(d, "theta"), p)
    res = _pcg_forms(An, p["m"] * _t(d, "v"), 1e-9, 100)
    assert res["colour"][:2] == res["gather"][:2] == res["fused"][:2] == (0, "negative_curvature")
    assert torch.equal(res["colour"][2], res["gather"][2])               # x = z = b / d at k = 0
    assert torch.equal(res["colour"][2], res["fused"][2])
    p2, A2, *_ = _linear_system()
    b2 = p2["m"] * torch.ones(A2.mesh.n_dof, dtype=torch.float64, device=DEV)
    cap = _pcg_forms(A2, b2, 1e-30, 7)
    assert cap["gather"][:2] == cap["fused"][:2] == (7, "max_iter")
    assert rel(cap["fused"][2], cap["colour"][2]) < 1e-10


@pytest.mark.parametrize("name", DEVICE_PRECONDITIONER_CASES)
@pytest.mark.parametrize("form", ["gather", "fused"])
def test_newton_solve_with_the_gather_form(name, form):
    d = load(name)
    p = params_from(d, DEV)
    th = _t(d, "theta")
    pre = str(d["preconditioner"]) if "preconditioner" in d else "jacobi"
    ws = NewtonWorkspace(p, pcg_form=form, preconditioner=pre)
    u, info = newton_krylov_solve(p, th, int(d["n_load_steps"]), float(d["tol"]), verbose=False, workspace=ws,
                                  preconditioner=pre)
    assert info["converged"] and rel(u, d["u_star"]) < 1e-9
    assert info["total_newton"] == int(d["total_newton"])


def test_reference_frame_pcg_matches_the_fp64_solution():
    p, A, M, A_ref, d_ref, b = _linear_system()
    u = torch.as_tensor(load("operator_quad4_h0.1_theta")["u"], device=DEV)
    th = torch.as_tensor(load("operator_quad4_h0.1_theta")["theta"], device=DEV)
    ws64 = NewtonWorkspace(p, "fp64")
    ws32 = NewtonWorkspace(p, "fp32")
    assert ws32.moduli_kind == "ref" and ws32.C.numel() == ws32.mesh.moduli_numel_ref()
    xs = {}
    for ws in (ws64, ws32):
        ws.set_theta(th)
        ws.linearize(u)
        ws.b.copy_(b)
        k, status = ws.pcg.solve(1e-10, 3000)
        assert status == "converged"
        xs[ws.precision] = ws.du.clone()
    assert rel(xs["fp32"], xs["fp64"]) < 1e-4                            # FP32 operator, FP64 recurrences
    assert torch.equal(ws32.diag, ws64.diag)                            # the diagonal is FP64 in both


# ------------------------------------------------------------------------------------------------
# nodal block-Jacobi (operators.py:586-625) inside the device PCG
# ------------------------------------------------------------------------------------------------
@pytest.mark.parametrize("form", ["colour", "gather", "fused"])
def test_block_jacobi_pcg_follows_the_reference_recurrences(form):
    from difffea_b200.operators import compute_block_jacobi
    d = load("operator_quad4_h0.1_theta")
    p = params_from(d, DEV)
    u, th = _t(d, "u"), _t(d, "theta")
    A = make_tangent_operator("cuda", u, th, p)
    blocks = compute_block_jacobi(u, th, p)
    b = p["m"] * _t(d, "v")
    bb, xx = b.clone(), torch.empty_like(b)
    solver = DevicePCG(A.mesh, A.C, blocks, bb, xx, form=form, preconditioner="block_jacobi")
    k, status = solver.solve(1e-10, 2000)
    solver.close()
    P = oracle.as_problem(p)
    x_ref, k_ref = oracle.pcg(oracle.make_operator("qp_ew", u.cpu(), th.cpu(), P), b.cpu(),
                              oracle.block_jacobi(u.cpu(), th.cpu(), P), rtol=1e-10, max_iter=2000)
    assert status == "converged" and abs(k - k_ref) <= 1 and rel(xx, x_ref) < 1e-9


def test_block_jacobi_mixed_precision_solve():
    p = build_rectangle_problem("quad9", 24, 12, 2.0, 1.0, E=1.0, nu=0.44, load=(0.0, -2e-3), device=DEV)
    th = torch.ones(p["conn"].shape[0], dtype=torch.float64, device=DEV)
    tol = 1e-11 * float(torch.norm(p["f"]))
    u_j, i_j = newton_krylov_solve(p, th, 2, tol, verbose=False, pcg_max_iter=5000)
    u_b, i_b = newton_krylov_solve(p, th, 2, tol, verbose=False, pcg_max_iter=5000, precision="fp32",
                                   preconditioner="block_jacobi")
    assert i_j["converged"] and i_b["converged"] and rel(u_b, u_j) < 1e-8


# ------------------------------------------------------------------------------------------------
# batched PCG: several solves advance together, bitwise as when each runs alone
# ------------------------------------------------------------------------------------------------
def _serving_system(et, nx, seed):
    from difffea_b200.serving import Request, request_problem
    p = request_problem(Request(seed, et, nx, 1.0 + 0.1 * seed, 0.3, 0.02), DEV, build_on_device=True)
    th = torch.ones(p["conn"].shape[0], dtype=torch.float64, device=DEV)
    ws = NewtonWorkspace(p, "fp32", use_graph=0, pcg_form="gather", max_blocks=64)
    ws.set_theta(th)
    g = torch.Generator().manual_seed(seed)
    u = (((torch.rand(p["f"].shape[0], dtype=torch.float64, generator=g) * 2 - 1) * 1e-3).to(DEV)) * p["m"]
    ws.linearize(u)
    b = p["m"] * torch.randn(p["f"].shape[0], dtype=torch.float64, generator=g).to(DEV)
    return ws, b


def test_batched_pcg_is_bitwise_the_solo_solve():
    import threading
    from difffea_b200.krylov import BatchExecutor
    cases = [("quad4", 64, 1, 1e-10, 5000), ("quad9", 32, 2, 1e-10, 5000), ("quad4", 128, 3, 1e-8, 60),
             ("quad9", 16, 4, 1e-12, 5000)]
    systems = [_serving_system(et, nx, seed) for et, nx, seed, _, _ in cases]
    solo = []
    for (ws, b), (_, _, _, rtol, cap) in zip(systems, cases):
        ws.b.copy_(b)
        k, status = ws.pcg.solve(rtol, cap)
        solo.append((k, status, ws.du.clone()))
    ex = BatchExecutor(DEV, capacity=4, max_blocks=64)
    out = [None] * len(cases)

    def run(i):
        ws, b = systems[i]
        torch.cuda.set_device(0)
        with torch.cuda.stream(torch.cuda.Stream()):
            ws.b.copy_(b)
            k, status = ex.solve(ws.pcg, cases[i][3], cases[i][4])
            out[i] = (k, status, ws.du.clone())

    threads = [threading.Thread(target=run, args=(i,)) for i in range(len(cases))]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    ex.close()
    assert ex.peak_batch >= 2
    for (k0, s0, x0), (k1, s1, x1) in zip(solo, out):
        assert (k0, s0) == (k1, s1)
        assert torch.equal(x0, x1)
    assert solo[2][:2] == (60, "max_iter")
