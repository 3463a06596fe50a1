"""
Boundary selection, DOF masks and consistent edge loads (host set-up).

Same semantics as the reference's builders (boundary_conditions.py:141-277): nodes on a side of the
bounding box within a relative tolerance; node-major DOFs (dof = 2 * node + component); boundary edges
are the edges that belong to exactly one element, kept in element order; a uniform traction whose
total is given is integrated against the edge shape functions with a 3-point Gauss rule (work-
equivalent nodal forces).
"""
import torch

from difffea_b200.elements import edge_shape_at_rule, gauss_1d


def bounding_box(nodes):
    """(lo, hi): the per-coordinate minima and maxima of the nodes, (2,) each."""
    return torch.aminmax(nodes, dim=0)


def select_boundary_nodes(nodes, side, tol=1e-6, box=None):
    """(N,) bool mask of the nodes on side "left" | "right" | "bottom" | "top" of the bounding box (``box``:
    ``bounding_box(nodes)``, when the caller has it already)."""
    if side not in ("left", "right", "bottom", "top"):
        raise ValueError("side must be 'left', 'right', 'bottom' or 'top'")
    lo, hi = bounding_box(nodes) if box is None else box
    eps = tol * (hi - lo).max()
    c = 0 if side in ("left", "right") else 1
    if side in ("left", "bottom"):
        return nodes[:, c] <= lo[c] + eps
    return nodes[:, c] >= hi[c] - eps


def dofs_from_node_mask(node_mask, components=(0, 1)):
    """Expand a node mask (N,) to a DOF mask (2N,) for the given components (0 = x, 1 = y)."""
    out = torch.zeros(node_mask.shape[0], 2, dtype=torch.bool, device=node_mask.device)
    for c in components:
        out[:, c] = node_mask
    return out.reshape(-1)


def boundary_edges(conn, edge_local_nodes, node_mask=None, n_nodes=None):
    """
    Edges used by exactly one element, as (E, k) global node ids [start, end(, mid)], element order.
    ``node_mask`` (N,) keeps only the edges whose nodes all lie in it; the two copies of an inner edge have
    the same nodes, so they pass or fail the mask together and counting among the kept edges gives the same
    boundary edges as counting among all.  ``n_nodes`` (more than the largest node id) spares reading that
    id back from the device.
    """
    k = len(edge_local_nodes[0])
    all_edges = conn[:, torch.tensor(edge_local_nodes, device=conn.device)].reshape(-1, k)
    if node_mask is not None:
        all_edges = all_edges[node_mask[all_edges].all(dim=1)]
    lo = torch.minimum(all_edges[:, 0], all_edges[:, 1])
    hi = torch.maximum(all_edges[:, 0], all_edges[:, 1])
    key = lo * (int(n_nodes) if n_nodes is not None else int(conn.max()) + 1) + hi
    _, inverse, counts = torch.unique(key, return_inverse=True, return_counts=True)
    return all_edges[counts[inverse] == 1]


def edge_traction_load(nodes, edges, order, node_mask, total_force, n_gauss=3):
    """
    Consistent nodal forces (N, 2) of a uniform traction of total (Fx, Fy) on the boundary edges whose
    nodes all lie in ``node_mask``; ``order`` is the edge interpolation order (1 or 2).
    """
    dtype, device = nodes.dtype, nodes.device
    f = torch.zeros_like(nodes)
    edges = edges[node_mask[edges].all(dim=1)]
    if edges.shape[0] == 0:
        return f
    s, w = gauss_1d(n_gauss, dtype, device)   # (host leggauss values moved to the device)
    N, dN = edge_shape_at_rule(order, s)                           # (g, k)
    Xe = nodes[edges]                                              # (E, k, 2)
    tangent = torch.einsum("gk,ekd->egd", dN, Xe)                  # dX/ds at every Gauss point
    speed = torch.linalg.norm(tangent, dim=-1)                     # (E, g)
    length = torch.einsum("eg,g->", speed, w)
    t = torch.as_tensor(total_force, dtype=dtype, device=device) / length
    f_edge = torch.einsum("g,ga,eg,i->eai", w, N, speed, t)        # (E, k, 2)
    f.index_add_(0, edges.reshape(-1), f_edge.reshape(-1, 2))
    return f
