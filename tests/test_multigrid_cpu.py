"""
Multigrid preconditioner, host side: the grid inference of structured meshes, and the oracle's V-cycle
(its CPU restatement) -- symmetric, and a mesh-independent number of PCG iterations.
"""
import pytest
import torch

import oracle
from oracle import multigrid as omg
from difffea_b200.mesh import create_quarter_plate_mesh, create_rectangle_mesh
from difffea_b200.multigrid import structured_grid
from difffea_b200.problem import build_rectangle_problem


@pytest.mark.parametrize("et,nx,ny", [("quad4", 7, 3), ("quad9", 4, 6), ("quad4", 1, 5)])
def test_grid_of_rectangle_meshes(et, nx, ny):
    nodes, conn = create_rectangle_mesh(et, 2.0, 1.0, nx, ny)
    g = structured_grid(conn, nodes.shape[0])
    span = 2 if et == "quad9" else 1
    assert (g["span"], g["ncx"], g["ncy"], g["gx"], g["gy"]) == (span, nx, ny, span * nx, span * ny)
    ij = g["node_ij"].long()
    assert torch.allclose(ij[:, 0].double() * 2.0 / (span * nx), nodes[:, 0], atol=1e-14)   # grid position = x
    assert torch.equal(g["gnode"].long()[ij[:, 0] * (span * ny + 1) + ij[:, 1]], torch.arange(nodes.shape[0]))


@pytest.mark.parametrize("et", ["quad4", "quad9"])
def test_grid_of_the_quarter_plate(et):
    nodes, conn = create_quarter_plate_mesh(et, 6, 4)
    g = structured_grid(conn, nodes.shape[0])
    assert g is not None and (g["ncx"], g["ncy"]) == (4, 6)                          # radial cells first


@pytest.mark.parametrize("et,span,epc", [("tri3", 1, 2), ("tri6", 2, 2), ("quad8", 2, 1)])
def test_grid_of_triangle_and_serendipity_meshes(et, span, epc):
    nodes, conn = create_rectangle_mesh(et, 2.0, 1.0, 5, 3)
    g = structured_grid(conn, nodes.shape[0])
    assert (g["span"], g["epc"], g["ncx"], g["ncy"]) == (span, epc, 5, 3)
    ij = g["node_ij"].double()
    assert torch.allclose(ij[:, 0] * 2.0 / (span * 5), nodes[:, 0], atol=1e-14)
    assert torch.allclose(ij[:, 1] / (span * 3), nodes[:, 1], atol=1e-14)
    if et == "quad8":                                   # the cell centres are not mesh nodes
        assert int((g["gnode"] < 0).sum()) == 15


def test_no_grid_for_shuffled_meshes():
    nodes, conn = create_rectangle_mesh("quad4", 1.0, 1.0, 4, 4)
    assert structured_grid(conn[torch.randperm(16, generator=torch.Generator().manual_seed(0))], 25) is None
    nodes, conn = create_rectangle_mesh("tri3", 1.0, 1.0, 4, 4)
    assert structured_grid(conn.flip(1), 25) is None


@pytest.mark.parametrize("et,nx,ny,rtol_it", [("quad4", 16, 4, 16), ("quad4", 33, 9, 16), ("quad9", 8, 2, 16)])
def test_oracle_vcycle_is_spd_and_converges_fast(et, nx, ny, rtol_it):
    p = build_rectangle_problem(et, nx, ny, 4.0, 1.0, load=(0.0, -0.01))
    P = oracle.as_problem(p)
    th = 0.5 + torch.rand(p["conn"].shape[0], dtype=torch.float64, generator=torch.Generator().manual_seed(1))
    u = torch.zeros(p["f"].numel(), dtype=torch.float64)
    span = 2 if et == "quad9" else 1
    M, levels, lams = omg.preconditioner(u, th, P, span * nx, span * ny, oracle.jacobi_diagonal(u, th, P))
    A = levels[0]["A"]
    g = torch.Generator().manual_seed(2)
    r1, r2 = torch.randn(A.shape[0], dtype=torch.float64, generator=g), torch.randn(A.shape[0], dtype=torch.float64, generator=g)
    assert abs(float(r2 @ M(r1) - r1 @ M(r2))) < 1e-12 * abs(float(r1 @ M(r1)))
    assert float(r1 @ M(r1)) > 0
    _, it = oracle.pcg(lambda v: A @ v, P["f"] * P["m"], M, rtol=1e-10, max_iter=500)
    assert it <= rtol_it
