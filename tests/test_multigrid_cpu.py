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


def test_lanczos_bound_is_the_largest_ritz_value():
    """The C++ set-up's bound (Sturm bisection on the CG tridiagonal) equals numpy's eigenvalue, on the CPU."""
    import ctypes
    import numpy as np
    from difffea_b200 import _lib
    lib = _lib.load()
    rng = np.random.default_rng(0)
    for steps in (1, 3, 10, 20):
        hist = np.empty(2 * steps)
        hist[0::2] = rng.uniform(0.3, 1.5, steps)          # alpha_k > 0
        hist[1::2] = rng.uniform(0.0, 0.9, steps)          # beta_k >= 0
        a, b = hist[0::2], hist[1::2]
        T = np.zeros((steps, steps))
        for k in range(steps):
            T[k, k] = 1 / a[k] + (b[k - 1] / a[k - 1] if k else 0.0)
            if k + 1 < steps:
                T[k, k + 1] = T[k + 1, k] = np.sqrt(b[k]) / a[k]
        got = lib.dfea_mg_lanczos_bound(hist.ctypes.data_as(ctypes.c_void_p), steps)
        assert abs(got - np.linalg.eigvalsh(T).max()) < 1e-12 * abs(got)
    # a breakdown (alpha <= 0) cuts the matrix; no valid step gives the default 2.5
    hist = np.array([0.5, 0.2, -1.0, 0.1])
    assert abs(lib.dfea_mg_lanczos_bound(hist.ctypes.data_as(ctypes.c_void_p), 2) - 2.0) < 1e-12
    assert lib.dfea_mg_lanczos_bound(np.array([np.nan, 0.0]).ctypes.data_as(ctypes.c_void_p), 1) == 2.5
    assert lib.dfea_mg_lanczos_bound(hist.ctypes.data_as(ctypes.c_void_p), 0) == -1.0


def test_grid_inference_over_random_meshes():
    """Every structured rectangle mesh (random element type and cell counts) is recognised with its exact
    counts and node positions; a mesh with two nodes swapped is not."""
    g = torch.Generator().manual_seed(3)
    spans = {"quad4": 1, "tri3": 1, "quad9": 2, "quad8": 2, "tri6": 2}
    for _ in range(25):
        et = ["quad4", "quad9", "quad8", "tri3", "tri6"][int(torch.randint(0, 5, (1,), generator=g))]
        nx, ny = (int(v) for v in torch.randint(1, 12, (2,), generator=g))
        nodes, conn = create_rectangle_mesh(et, float(nx), float(ny), nx, ny)
        grid = structured_grid(conn, nodes.shape[0])
        assert grid is not None and (grid["ncx"], grid["ncy"]) == (nx, ny), (et, nx, ny)
        span = spans[et]
        assert torch.allclose(grid["node_ij"].double() / span, nodes, atol=1e-12)
        if conn.shape[0] > 1:
            bad = conn.clone()
            bad[0, 0], bad[0, 1] = conn[0, 1], conn[0, 0]
            assert structured_grid(bad, nodes.shape[0]) is None
