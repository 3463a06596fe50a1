"""
Parity at the sizes the benchmark configurations state, against the oracle (the CPU restatement of the
reference's algorithm, pinned to the reference's own outputs by tests/test_oracle_golden.py).

    plain solve      100 x 100 Q4 unit square, E = 1, nu = 0.3, traction (0.1, 0) on the right edge, left
                     edge clamped, 3 load steps, Newton tol 1e-10: the complete FP64 solve against the
                     oracle's (tangent "qp", Jacobi-PCG, newton_krylov.py:185-264), Newton and CG counts
    tangent product  structured Q4 and Q9, n x n unit cells, u = m * U(-0.05, 0.05), v ~ N(0, 1) from one
                     generator seeded 0, theta = 1: moduli, the FP64 product (bar 1e-11, the reference's
                     qp_ew, operators.py:385-412) and the Jacobi diagonal against the oracle on the whole mesh
                     at 40k / 160k elements (and 640k Q4), the FP32-moduli products within their FP32 bars;
                     at 640k Q9 and 2.56M Q4 / Q9 elements the product rows of a seeded sample of nodes
                     against the oracle evaluated on those nodes' element patches (a row of A(v) depends only
                     on the elements around its node, so this is the same check, exact at any mesh size)
    quarter plate    the mapped 256 x 256 Q9 plate (5 load steps): the FP64 and FP32-operator solutions
                     satisfy the oracle's equilibrium equations to the solve tolerance, and the strain energy
                     agrees with the oracle's at the same state
    serving          requests of the seeded stream with nx >= 256 (Q4 and Q9), served by the engine (FP32
                     operator, multigrid-preconditioned PCG, FP64 Newton), against the oracle's complete solve
                     with the reference's ILU-preconditioned PCG (operators.py:680-699), bar 1e-8
"""
import pytest
import torch

import oracle
from difffea_b200.newton_krylov import newton_krylov_solve
from difffea_b200.operators import global_residual, make_A_operator_cuda, make_tangent_operator, strain_energy
from difffea_b200.problem import build_quarter_plate_problem, build_rectangle_problem
from golden_utils import rel

pytestmark = pytest.mark.gpu
DEV = "cuda"


def unpack_moduli(mesh, C):
    """(n_el, n_q, 4, 4) in original element order from the colour-sorted FP64 SoA layout of kernel (a)."""
    S, nq, n = mesh.stride, mesh.n_q, mesh.n_el
    slot = C.view(nq, 8, S, 2)[:, :, :n, :].permute(2, 0, 1, 3).reshape(n, nq, 4, 4)
    out = torch.empty_like(slot)
    out[mesh.perm] = slot
    return out


def config2_state(et, n):
    """The tangent-product benchmark's inputs: n x n cells of unit size, seeded state and input vector."""
    p = build_rectangle_problem(et, n, n, float(n), float(n), E=1.0, nu=0.3, device=DEV, build_on_device=True)
    g = torch.Generator().manual_seed(0)
    N2 = p["f"].shape[0]
    u = (((torch.rand(N2, dtype=torch.float64, generator=g) * 2 - 1) * 0.05).to(DEV)) * p["m"]
    v = torch.randn(N2, dtype=torch.float64, generator=g).to(DEV)
    th = torch.ones(p["conn"].shape[0], dtype=torch.float64, device=DEV)
    return p, u, v, th


# ---------------------------------------------------------------------------------------------
# plain solve
# ---------------------------------------------------------------------------------------------
def test_plain_100x100_solve_against_the_oracle():
    p = build_rectangle_problem("quad4", 100, 100, 1.0, 1.0, E=1.0, nu=0.3, load=(0.1, 0.0), device=DEV)
    th = torch.ones(p["conn"].shape[0], dtype=torch.float64, device=DEV)
    u, info = newton_krylov_solve(p, th, 3, 1e-10, verbose=False)
    u_ref, info_ref = oracle.newton_krylov_solve(oracle.as_problem(p), th.cpu(), 3, 1e-10, tangent="qp")
    err = rel(u, u_ref)
    print(f"\nplain 100x100 Q4: rel err {err:.2e}; Newton {info['total_newton']} (oracle {info_ref['total_newton']}), "
          f"CG {info['total_cg']} (oracle {info_ref['total_cg']}), max u_x {float(u[0::2].max()):.4f}")
    assert info["converged"] and info_ref["converged"]
    assert err <= 1e-9                                      # the parity bar for complete solutions
    assert info["total_newton"] == info_ref["total_newton"]
    assert abs(info["total_cg"] - info_ref["total_cg"]) <= 0.01 * info_ref["total_cg"]
    assert 0.09 < float(u[0::2].max()) < 0.10               # ~10 % stretch


# ---------------------------------------------------------------------------------------------
# tangent product
# ---------------------------------------------------------------------------------------------
@pytest.mark.parametrize("et,n", [("quad4", 200), ("quad9", 200), ("quad4", 400), ("quad9", 400), ("quad4", 800)])
def test_product_moduli_and_diagonal_against_the_oracle(et, n):
    p, u, v, th = config2_state(et, n)
    A = make_tangent_operator("cuda", u, th, p)
    y = A(v)
    P = oracle.as_problem(p)
    uc, thc, vc = u.cpu(), th.cpu(), v.cpu()
    C_ref = oracle.moduli(uc, thc, P)
    y_ref = oracle.apply_qp_ew(C_ref, vc, P)
    e_y, e_C = rel(y, y_ref), rel(unpack_moduli(A.mesh, A.C), C_ref)
    e_d = rel(A.diag, oracle.jacobi_diagonal(uc, thc, P))
    # FP32 moduli (and gradients) applied to FP64 vectors in FP64 arithmetic, and to FP32 vectors
    A32 = make_A_operator_cuda(u, th, p, precision="fp32")
    e_mixed, e_f32 = rel(A32(v), y_ref), rel(A32(v.float()), y_ref)
    print(f"\n{et} {p['conn'].shape[0]} el: product {e_y:.1e}, moduli {e_C:.1e}, diag {e_d:.1e}, "
          f"fp32 moduli on f64 vectors {e_mixed:.1e}, all fp32 {e_f32:.1e}")
    assert e_y < 1e-11 and e_C < 1e-12 and e_d < 1e-12
    assert e_mixed < 2e-6 and e_f32 < 2e-5


def oracle_rows(p, u, v, th, node_ids):
    """
    (DOF ids, y at those DOFs, element ids, moduli of those elements) of the oracle's qp_ew product restricted
    to the rows of ``node_ids``: computed on the patch of elements incident to those nodes, with the full
    state and input vector on the patch's nodes.
    """
    conn = p["conn"].cpu()
    node_ids = torch.unique(node_ids.cpu())
    els = torch.nonzero(torch.isin(conn, node_ids).any(1)).squeeze(1)
    local_nodes, inv = torch.unique(conn[els], return_inverse=True)
    dofs = (2 * local_nodes[:, None] + torch.arange(2)).reshape(-1)
    P = oracle.as_problem({"nodes": p["nodes"][local_nodes.to(DEV)], "conn": inv.reshape(els.numel(), -1),
                           "dN_dX": p["dN_dX"][els.to(DEV)], "w_detJ": p["w_detJ"][els.to(DEV)],
                           "f": torch.zeros(dofs.numel(), dtype=torch.float64), "m": p["m"].cpu()[dofs],
                           "u_D": torch.zeros(dofs.numel(), dtype=torch.float64), "fixed": p["fixed"].cpu()[dofs],
                           "mat_p": p["mat_p"], "mat_scalable": p["mat_scalable"],
                           "material": p.get("material", "neo_hookean")})
    C = oracle.moduli(u.cpu()[dofs], th.cpu()[els], P)
    y_local = oracle.apply_qp_ew(C, v.cpu()[dofs], P)
    rows = (2 * torch.searchsorted(local_nodes, node_ids)[:, None] + torch.arange(2)).reshape(-1)
    return (2 * node_ids[:, None] + torch.arange(2)).reshape(-1), y_local[rows], els, C


@pytest.mark.parametrize("et,n", [("quad9", 800), ("quad4", 1600), ("quad9", 1600)])
def test_product_rows_at_full_size_against_the_oracle(et, n):
    p, u, v, th = config2_state(et, n)
    A = make_tangent_operator("cuda", u, th, p)
    y = A(v)
    N = p["nodes"].shape[0]
    g = torch.Generator().manual_seed(1)
    sample = torch.cat([torch.randint(0, N, (512,), generator=g),
                        torch.tensor([0, N - 1, n // 2, N // 2])])          # corners (fixed edge), a mid node
    dofs, y_ref, els, C_ref = oracle_rows(p, u, v, th, sample)
    e_y = rel(y.cpu()[dofs], y_ref)
    e_C = rel(unpack_moduli(A.mesh, A.C)[els.to(DEV)], C_ref)
    print(f"\n{et} {p['conn'].shape[0]} el: {dofs.numel()} rows of A(v) {e_y:.1e}, moduli of {els.numel()} "
          f"elements {e_C:.1e}")
    assert e_y < 1e-11 and e_C < 1e-12


# ---------------------------------------------------------------------------------------------
# quarter plate
# ---------------------------------------------------------------------------------------------
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_quarter_plate_256_satisfies_the_oracle_equilibrium(precision):
    p = build_quarter_plate_problem("quad9", 256, 256, radius=1.0, half_width=10.0, traction=0.1, device=DEV)
    th = torch.ones(p["conn"].shape[0], dtype=torch.float64, device=DEV)
    fn = float(torch.norm(p["f"]))
    tol = 1e-11 * fn
    u, info = newton_krylov_solve(p, th, 5, tol, verbose=False, pcg_max_iter=20000, precision=precision,
                                  preconditioner="multigrid")
    assert info["converged"]
    P = oracle.as_problem(p)
    uc, thc = u.cpu(), th.cpu()
    R_ref = oracle.residual(uc, thc, P, 1.0)
    r_ref, r_gpu = float(torch.norm(R_ref)), float(torch.norm(global_residual(u, th, p)))
    W, W_ref = float(strain_energy(u, th, p)), float(oracle.strain_energy(uc, thc, P))
    print(f"\nplate 256x256 Q9 {precision}: oracle ||R(u)|| = {r_ref:.2e} ({r_ref / fn:.1e} ||f||), device "
          f"{r_gpu:.2e}; energy {W:.12e} vs oracle {W_ref:.12e}")
    assert r_ref < 1e-10 * fn                              # the reference's equations hold at the device solution
    assert abs(W - W_ref) <= 1e-12 * abs(W_ref)


# ---------------------------------------------------------------------------------------------
# serving requests at nx >= 256
# ---------------------------------------------------------------------------------------------
def _big_requests():
    from difffea_b200.serving import request_stream
    reqs = request_stream(2000, seed=0)
    out = []
    for et in ("quad4", "quad9"):
        cands = sorted((r for r in reqs if r.element_type == et and r.nx >= 256), key=lambda r: (r.nx, r.rid))
        out += cands[:1]
    return out


def test_serving_requests_nx256_plus_against_the_oracle():
    from difffea_b200.serving import ServingEngine, reference_request_problem
    reqs = _big_requests()
    eng = ServingEngine(n_slots=4, device=DEV, precision="fp32")
    results = eng.run(reqs)
    for r, res in zip(reqs, results):
        assert res.converged and not res.error, res.error
        p = reference_request_problem(r)           # the oracle's input: built independently of the library
        P = oracle.as_problem(p)
        tol = 1e-10 * float(torch.linalg.vector_norm(p["f"]))
        th = torch.ones(p["conn"].shape[0], dtype=torch.float64)
        u_ref, info = oracle.newton_krylov_solve(P, th, 1, tol, tangent="qp", pcg_max_iter=5000, precond="ilu")
        assert info["converged"]
        err = rel(res.u, u_ref)
        print(f"\nrequest {r.rid} {r.element_type} nx={r.nx} ({r.n_nodes} nodes): engine vs oracle {err:.2e}; "
              f"Newton {res.newton} (oracle {info['total_newton']}), CG {res.cg}")
        assert err <= 1e-8
