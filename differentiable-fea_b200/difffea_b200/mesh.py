"""
Structured meshes of a rectangle and the mapped quarter plate with a hole.

Rectangle meshes reproduce the reference's numbering exactly (mesh.py:19-438), because identical inputs
are what parity is checked on: grid nodes are numbered x-major, id = i * (n_y + 1) + j for grid column i
and row j; cells are numbered x-major as well, cell (i, j) -> i * ny + j; local node orders are those of
the element library; a triangle mesh lists all lower-left triangles of the cells first, then all
upper-right ones.  Coordinates come from torch.linspace so that they agree bit for bit.

``create_quarter_plate_mesh`` has no reference counterpart (the reference meshes that geometry with
Gmsh, which is not available here): it maps a structured Q9/Q4 grid onto the quarter of a square plate
with a circular hole, graded towards the hole.
"""
import math

import torch


def _grid(Lx, Ly, gx, gy, dtype, device):
    x = torch.linspace(0.0, Lx, gx + 1, dtype=dtype, device=device)
    y = torch.linspace(0.0, Ly, gy + 1, dtype=dtype, device=device)
    X = x[:, None].expand(gx + 1, gy + 1)
    Y = y[None, :].expand(gx + 1, gy + 1)
    nodes = torch.stack([X.reshape(-1), Y.reshape(-1)], dim=1)
    ids = torch.arange((gx + 1) * (gy + 1), device=device).reshape(gx + 1, gy + 1)
    return nodes, ids


def _quad4_conn(ids, nx, ny):
    c = [ids[:nx, :ny], ids[1:nx + 1, :ny], ids[1:nx + 1, 1:ny + 1], ids[:nx, 1:ny + 1]]
    return torch.stack([t.reshape(-1) for t in c], dim=1)


def _quad9_conn(ids, nx, ny):
    # grid offsets (di, dj) of the nine local nodes inside a 2x2 block of grid cells
    offs = [(0, 0), (2, 0), (2, 2), (0, 2), (1, 0), (2, 1), (1, 2), (0, 1), (1, 1)]
    cols = [ids[di:di + 2 * nx:2, dj:dj + 2 * ny:2].reshape(-1) for di, dj in offs]
    return torch.stack(cols, dim=1)


def create_rectangle_mesh(element_type, Lx, Ly, nx, ny, dtype=torch.float64, device="cpu"):
    """Structured mesh of [0, Lx] x [0, Ly] with nx x ny cells -> (nodes (N, 2), conn (n_el, nen) int64)."""
    if element_type == "quad4":
        nodes, ids = _grid(Lx, Ly, nx, ny, dtype, device)
        return nodes, _quad4_conn(ids, nx, ny)
    if element_type in ("quad9", "tri6", "quad8"):
        nodes, ids = _grid(Lx, Ly, 2 * nx, 2 * ny, dtype, device)
        q9 = _quad9_conn(ids, nx, ny)
        if element_type == "quad9":
            return nodes, q9
        if element_type == "tri6":
            lower = q9[:, [0, 1, 3, 4, 8, 7]]
            upper = q9[:, [1, 2, 3, 5, 6, 8]]
            return nodes, torch.cat([lower, upper], dim=0)
        # quad8: drop the cell centres and renumber the remaining grid nodes consecutively
        keep = torch.ones(2 * nx + 1, 2 * ny + 1, dtype=torch.bool, device=device)
        keep[1:2 * nx:2, 1:2 * ny:2] = False
        keep = keep.reshape(-1)
        new_id = torch.full((keep.numel(),), -1, dtype=torch.int64, device=device)
        new_id[keep] = torch.arange(int(keep.sum()), device=device)
        return nodes[keep], new_id[q9[:, :8]]
    if element_type == "tri3":
        nodes, ids = _grid(Lx, Ly, nx, ny, dtype, device)
        q4 = _quad4_conn(ids, nx, ny)
        return nodes, torch.cat([q4[:, [0, 1, 3]], q4[:, [1, 2, 3]]], dim=0)
    raise ValueError(f"Unknown element type '{element_type}'. Choose one of "
                     f"['quad4', 'quad8', 'quad9', 'tri3', 'tri6'].")


def create_quarter_plate_mesh(element_type="quad9", n_theta=256, n_radial=256, radius=1.0, half_width=10.0,
                              grading=3.0, dtype=torch.float64, device="cpu"):
    """
    Mapped mesh of the quarter plate {0 <= x, y <= W} minus the disk r < R (W = half_width, R = radius).

    The logical grid (theta, s) in [0, pi/2] x [0, 1] is mapped to
        X(theta, s) = P_hole(theta) + s_g (P_edge(theta) - P_hole(theta)),
        P_hole = R (cos theta, sin theta),   P_edge = the ray's exit point on the square's outer edges,
        s_g = (exp(grading * s) - 1) / (exp(grading) - 1)      (cells cluster at the hole),
    and cut into n_theta x n_radial cells (Q9: 3x3 nodes per cell on the mapped coordinates, so edges are
    curved and the hole is represented to quadratic order).  Cells are numbered ring by ring outwards
    (radial index major); local node orders follow the element library with counter-clockwise corners.

    Returns (nodes (N, 2), conn (n_el, nen)).  The hole is at the origin, x = 0 and y = 0 are the
    symmetry lines, x = W is the loaded edge.
    """
    if element_type not in ("quad9", "quad4"):
        raise ValueError("the quarter-plate mesher builds quad9 or quad4 meshes")
    k = 2 if element_type == "quad9" else 1
    gt, gs = k * n_theta, k * n_radial
    t = torch.linspace(0.0, 0.5 * math.pi, gt + 1, dtype=dtype, device=device)
    s = torch.linspace(0.0, 1.0, gs + 1, dtype=dtype, device=device)
    sg = torch.expm1(grading * s) / math.expm1(grading) if grading > 0 else s
    ct, st = torch.cos(t), torch.sin(t)
    hole = torch.stack([radius * ct, radius * st], dim=1)                       # (gt+1, 2)
    # exit point of the ray at angle t on the outer square edges x = W (t <= pi/4) or y = W
    on_right = t <= 0.25 * math.pi + 1e-15
    edge = torch.where(on_right[:, None],
                       torch.stack([torch.full_like(t, half_width), half_width * torch.tan(torch.clamp(t, max=0.25 * math.pi))], 1),
                       torch.stack([half_width * ct / torch.clamp(st, min=1e-300), torch.full_like(t, half_width)], 1))
    edge[0] = torch.tensor([half_width, 0.0], dtype=dtype, device=device)
    edge[-1] = torch.tensor([0.0, half_width], dtype=dtype, device=device)
    idx = gt // 2
    if gt % 2 == 0:
        edge[idx] = torch.tensor([half_width, half_width], dtype=dtype, device=device)
    X = hole[:, None, :] + sg[None, :, None] * (edge - hole)[:, None, :]       # (gt+1, gs+1, 2)
    X[0, :, 1] = 0.0                                                           # exact symmetry lines
    X[-1, :, 0] = 0.0
    nodes = X.reshape(-1, 2)
    ids = torch.arange((gt + 1) * (gs + 1), device=device).reshape(gt + 1, gs + 1)
    # grid axis 0 is theta (counter-clockwise about the hole), axis 1 is s (outwards).  A cell's local
    # xi runs along s and eta along theta, which makes the corner order (s, theta) counter-clockwise.
    idsT = ids.transpose(0, 1)                                                # [s, theta]
    if element_type == "quad4":
        conn = _quad4_conn(idsT, n_radial, n_theta)
    else:
        conn = _quad9_conn(idsT, n_radial, n_theta)
    return nodes, conn.contiguous()
