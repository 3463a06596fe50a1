"""
Geometric multigrid preconditioner on the GPU: one V-cycle against the oracle's dense restatement (odd and
even grids, Q4 and Q9, clamped and roller supports, non-uniform theta, physical and reference-frame FP32
moduli), complete solves against the reference's solutions, mesh-independent iteration counts, and
the mapped quarter-plate grid.  A V-cycle agrees with the oracle to 1e-10 (the two assemble the coarse
operators in different orders and invert the coarsest one differently); solutions to 1e-9 as elsewhere.
"""
import pytest
import torch

import oracle
from oracle import multigrid as omg
from difffea_b200 import _lib
from difffea_b200.multigrid import Multigrid
from difffea_b200.newton_krylov import newton_krylov_solve
from difffea_b200.operators import make_A_operator_cuda, make_preconditioner
from difffea_b200.cuda_mesh import cuda_mesh
from difffea_b200.problem import build_quarter_plate_problem, build_rectangle_problem
from difffea_b200.workspace import NewtonWorkspace
from golden_utils import load, params_from, rel

pytestmark = pytest.mark.gpu
DEV = "cuda"


def _state(p, seed, amp):
    g = torch.Generator().manual_seed(seed)
    n, n_el = p["f"].numel(), p["conn"].shape[0]
    u = (amp * torch.randn(n, dtype=torch.float64, generator=g)).to(DEV) * p["m"]
    th = (0.5 + torch.rand(n_el, dtype=torch.float64, generator=g)).to(DEV)
    r = torch.randn(n, dtype=torch.float64, generator=g).to(DEV)
    return u, th, r


@pytest.mark.parametrize("et,nx,ny,fixed_dofs", [("quad4", 16, 4, "xy"), ("quad4", 13, 5, "xy"), ("quad4", 21, 3, "x"),
                                                  ("quad9", 6, 3, "xy"), ("quad9", 5, 2, "xy"), ("quad8", 6, 3, "xy"),
                                                  ("tri3", 13, 5, "xy"), ("tri6", 5, 3, "xy")])
def test_vcycle_matches_the_oracle(et, nx, ny, fixed_dofs):
    p = build_rectangle_problem(et, nx, ny, 4.0, 1.0, load=(0.0, -0.01), fixed_dofs=fixed_dofs, device=DEV)
    if fixed_dofs == "x":                                  # rollers on x = 0 plus one pinned corner in y
        p["fixed"][1] = True
        p["m"] = torch.where(p["fixed"], 0.0, 1.0).to(torch.float64)
    u, th, r = _state(p, 3, 0.01 * 4.0 / nx)
    z = make_preconditioner("multigrid", u, th, p)(r)
    P = oracle.as_problem(p)
    span = 2 if et in ("quad9", "quad8", "tri6") else 1
    uc, thc = u.cpu(), th.cpu()
    gx, gy = span * nx, span * ny                          # grid positions from the coordinates (4 x 1 domain)
    node_ij = torch.stack([torch.round(P["nodes"][:, 0] / 4.0 * gx), torch.round(P["nodes"][:, 1] * gy)], 1).long()
    M, levels, lams = omg.preconditioner(uc, thc, P, gx, gy, oracle.jacobi_diagonal(uc, thc, P), node_ij)
    z_ref = M(r.cpu())
    assert rel(z, z_ref) < 1e-10


@pytest.mark.parametrize("moduli", ["f32", "ref"])
def test_vcycle_from_fp32_moduli(moduli):
    """Level 1 from FP32 physical or reference-frame moduli: the cycle of the rounded operator."""
    p = build_rectangle_problem("quad9", 8, 4, 4.0, 1.0, load=(0.0, -0.01), device=DEV)
    u, th, r = _state(p, 4, 0.005)
    A = make_A_operator_cuda(u, th, p)
    mesh = cuda_mesh(p)
    mg64 = Multigrid(mesh, p)
    mg64.setup(A.C, _lib.DFEA_F64, A.diag)
    z64 = mg64(r)
    ws = NewtonWorkspace(p, "fp32", fp32_moduli="ref" if moduli == "ref" else "physical", preconditioner="multigrid")
    ws.set_theta(th)
    ws.linearize(u)
    z32 = ws.mg(r)
    assert rel(z32, z64) < 1e-5


@pytest.mark.parametrize("name", ["solve_quad4_h0.25_cantilever", "solve_quad9_h0.5_cantilever", "solve_quad4_h0.2_tension",
                                  "solve_tri6_h0.5_cantilever", "material_solve_fiber_reinforced_quad4_h0.5"])
def test_multigrid_solves_match_reference(name):
    d = load(name)
    p = params_from(d, DEV)
    th = torch.as_tensor(d["theta"], device=DEV)
    u, info = newton_krylov_solve(p, th, int(d["n_load_steps"]), float(d["tol"]), verbose=False,
                                  preconditioner="multigrid")
    assert info["converged"]
    assert rel(u, d["u_star"]) < 1e-9


def test_iterations_do_not_grow_with_the_mesh():
    """Linear solve of a 4:1 cantilever to 1e-8: multigrid iterations stay flat, Jacobi's grow with n."""
    its = {}
    for n in (32, 128, 512):
        p = build_rectangle_problem("quad4", n, n // 4, 4.0, 1.0, load=(0.0, -0.001), device=DEV, build_on_device=True)
        th = torch.ones(p["conn"].shape[0], dtype=torch.float64, device=DEV)
        u = torch.zeros_like(p["f"])
        for pre in ("multigrid", "jacobi"):
            ws = NewtonWorkspace(p, preconditioner=pre)
            ws.set_theta(th)
            ws.linearize(u)
            _, k, status = ws.solve(-p["f"] * p["m"], 1e-8, 20000)
            assert status == "converged"
            its[(pre, n)] = k
    print("\nPCG iterations to 1e-8:", its)
    assert max(its[("multigrid", n)] for n in (32, 128, 512)) <= 1.5 * its[("multigrid", 32)] + 2
    assert its[("jacobi", 512)] > 8 * its[("multigrid", 512)]


def test_quarter_plate_grid_and_mixed_precision():
    """The mapped quarter plate (transposed node numbering), Q9 32 x 32, FP32 operator + multigrid vs FP64 Jacobi."""
    p = build_quarter_plate_problem("quad9", 32, 32, radius=1.0, half_width=10.0, traction=0.1, device=DEV)
    th = torch.ones(p["conn"].shape[0], dtype=torch.float64, device=DEV)
    tol = 1e-11 * float(torch.norm(p["f"]))
    u_j, i_j = newton_krylov_solve(p, th, 5, tol, verbose=False, pcg_max_iter=20000)
    u_m, i_m = newton_krylov_solve(p, th, 5, tol, verbose=False, pcg_max_iter=20000, precision="fp32",
                                   preconditioner="multigrid")
    assert i_j["converged"] and i_m["converged"]
    print(f"\nplate 32x32 Q9: PCG iterations jacobi {i_j['total_cg']}, multigrid {i_m['total_cg']}")
    assert rel(u_m, u_j) < 1e-8
    assert i_m["total_cg"] * 5 < i_j["total_cg"]


def test_cycle_and_pcg_are_deterministic_across_linearisations():
    """The C++ driver's set-up, cycle and PCG give bit-identical results when repeated, at several states."""
    p = build_rectangle_problem("quad4", 24, 6, 4.0, 1.0, load=(0.0, -0.01), device=DEV)
    th = torch.ones(p["conn"].shape[0], dtype=torch.float64, device=DEV)
    ws = NewtonWorkspace(p, preconditioner="multigrid")
    ws.set_theta(th)
    r = torch.randn(p["f"].numel(), dtype=torch.float64, generator=torch.Generator().manual_seed(7)).to(DEV)
    for amp in (0.0, 0.002, 0.005):                        # random states well below h = 1/6 (no inversion)
        u, _, _ = _state(p, 11, amp) if amp else (torch.zeros_like(r), None, None)
        out = []
        for _ in range(2):
            ws.linearize(u)
            lams = [lv.lam for lv in ws.mg.levels[:-1]]
            z = ws.mg(r)
            du, it, status = ws.solve(-r, 1e-9, 200)
            out.append((lams, z, du.clone(), it, status))
        assert out[0][0] == out[1][0] and all(1.5 < x < 3.0 for x in out[0][0])
        assert torch.isfinite(out[0][1]).all() and torch.equal(out[0][1], out[1][1])
        assert torch.equal(out[0][2], out[1][2]) and out[0][3] == out[1][3] and out[0][4] == "converged"


def test_unstructured_mesh_is_refused():
    d = load("operator_quad4_h0.5_unit")
    p = params_from(d, DEV)
    perm = torch.randperm(p["conn"].shape[0], generator=torch.Generator().manual_seed(0)).to(DEV)
    p = dict(p, conn=p["conn"][perm], dN_dX=p["dN_dX"][perm], w_detJ=p["w_detJ"][perm])
    th = torch.ones(p["conn"].shape[0], dtype=torch.float64, device=DEV)
    with pytest.raises(ValueError, match="structured"):
        NewtonWorkspace(p, preconditioner="multigrid")


def test_preconditioner_closures_at_different_states_stay_independent():
    """Two make_preconditioner("multigrid") closures of one mesh share its hierarchy's buffers; the first still
    applies its own linearisation after the second has been set up (it sets the hierarchy up again)."""
    p = build_rectangle_problem("quad4", 32, 8, 4.0, 1.0, load=(0.0, -0.01), device=DEV)
    u1, th, r = _state(p, 21, 0.002)
    u2, _, _ = _state(p, 22, 0.004)
    M1 = make_preconditioner("multigrid", u1, th, p)
    z1 = M1(r).clone()
    M2 = make_preconditioner("multigrid", u2, th, p)
    z2 = M2(r).clone()
    assert M1.mg is M2.mg and not torch.equal(z1, z2)
    assert torch.equal(M1(r), z1)                          # re-set-up at u1: the same cycle, bit for bit
    assert torch.equal(M2(r), z2)


@pytest.mark.parametrize("et,code", [("quad4", "f64"), ("quad9", "f32ref")])
def test_graph_driven_hierarchy_matches_the_host_driven_one_bit_for_bit(et, code):
    """Set-ups replayed from a captured graph and the device-side PCG loop give the host-driven iterates: the
    same smoother bounds, solutions and iteration counts over several linearisations and solves (the first
    set-up and solve run directly, the second capture, the later ones replay)."""
    p = build_rectangle_problem(et, 48, 12, 4.0, 1.0, load=(0.02, 0.0), device=DEV)
    mesh = cuda_mesh(p)
    if code == "f32ref":
        mesh.ensure_ref_frame()
    hosted, graphed = Multigrid(mesh, p, graphs=False), Multigrid(mesh, p, graphs=True)
    n = mesh.n_dof
    b = torch.empty(n, dtype=torch.float64, device=DEV)
    xs = [torch.empty(n, dtype=torch.float64, device=DEV) for _ in range(2)]
    ws = NewtonWorkspace(p, "fp32" if code == "f32ref" else "fp64", preconditioner="jacobi")
    for step in range(4):
        u, th, r = _state(p, 40 + step, 0.01 * 4.0 / 48)
        ws.set_theta(th)
        ws.linearize(u)                                   # moduli and diagonal at this state
        b.copy_(r * p["m"])
        out = []
        for mg, x in zip((hosted, graphed), xs):
            mg.setup(ws.C, ws.moduli_code, ws.diag)
            k, status = mg.pcg(b, x, 1e-10, 200)
            out.append((k, status, [lv.lam for lv in mg.levels[:-1]]))
        assert out[0] == out[1] and out[0][1] == "converged"
        assert torch.equal(xs[0], xs[1])
    assert graphed.h.graphs and not hosted.h.graphs
    graphed.close()
    assert not graphed.h.graphs


@pytest.mark.parametrize("name", ["solve_quad4_h0.25_cantilever", "solve_quad9_h0.5_cantilever"])
def test_kept_smoother_bounds_still_reach_the_reference_solution(name):
    """Smoother bounds estimated at the first set-up only (bounds_every large): the later set-ups rebuild the
    coarse operators but keep lambda_max, and the Newton solve still meets the reference's solution."""
    d = load(name)
    p = params_from(d, DEV)
    th = torch.as_tensor(d["theta"], dtype=torch.float64, device=DEV)
    ws = NewtonWorkspace(p, preconditioner="multigrid", mg_bounds_every=1000)
    seen = []
    setup = ws.mg.setup

    def record(C, code, diag):
        setup(C, code, diag)
        seen.append([lv.lam for lv in ws.mg.levels[:-1]])
    ws.mg.setup = record
    u, info = newton_krylov_solve(p, th, int(d["n_load_steps"]), float(d["tol"]), verbose=False, workspace=ws,
                                  preconditioner="multigrid")
    assert info["converged"] and rel(u, d["u_star"]) < 1e-9
    assert len(seen) >= 2 and all(s == seen[0] for s in seen)
    assert ws.mg.h.setups == len(seen)


@pytest.mark.parametrize("name,graphs", [("solve_quad4_h0.25_cantilever", False), ("solve_quad9_h0.5_cantilever", True),
                                         ("solve_tri6_h0.5_cantilever", True)])
def test_gather_form_level0_products_reach_the_reference_solution(name, graphs):
    """The hierarchy's level-0 products in the gather form (element pass + node sums), host- or graph-driven:
    the Newton solve meets the reference's solution, and one V-cycle agrees with the colour form's to rounding."""
    d = load(name)
    p = params_from(d, DEV)
    th = torch.as_tensor(d["theta"], dtype=torch.float64, device=DEV)
    ws = NewtonWorkspace(p, preconditioner="multigrid", mg_gather=True, mg_graphs=graphs)
    u, info = newton_krylov_solve(p, th, int(d["n_load_steps"]), float(d["tol"]), verbose=False, workspace=ws,
                                  preconditioner="multigrid")
    assert info["converged"] and rel(u, d["u_star"]) < 1e-9
    colour = Multigrid(ws.mesh, p, graphs=False)
    colour.setup(ws.C, ws.moduli_code, ws.diag)
    r = torch.randn(ws.mesh.n_dof, dtype=torch.float64, generator=torch.Generator().manual_seed(9)).to(DEV)
    assert rel(ws.mg(r), colour(r)) < 1e-12
