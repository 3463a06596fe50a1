"""
Element library: node counts, quadrature rules, shape functions and their reference gradients.

The table follows the reference's element library (elements.py:38-58): the same five element types,
the same local node orderings (corners counter-clockwise first, then mid-sides, then the Q9 centre),
the same default quadrature (Q4 2x2 Gauss, Q8/Q9 3x3 Gauss, Tri3 centroid, Tri6 the 6-point degree-4
rule) and the same point ordering, so that Gauss-point arrays line up entry by entry with the
reference's.  Gradients are written in closed form (the reference obtains them with jacfwd,
grad_shape_functions_2d.py:47-64).

All functions here run on the host (set-up work); the kernels consume the tables they produce.
"""

import numpy as np
import torch

# name -> nen, n_corners, family, order, edges (local ids, [start, end(, mid)], CCW), quadrature
ELEMENT_LIBRARY = {
    "quad4": dict(n_nodes=4, n_corners=4, family="quad", order=1,
                  edges=[(0, 1), (1, 2), (2, 3), (3, 0)], gauss=("tensor", 2)),
    "quad8": dict(n_nodes=8, n_corners=4, family="quad", order=2,
                  edges=[(0, 1, 4), (1, 2, 5), (2, 3, 6), (3, 0, 7)], gauss=("tensor", 3)),
    "quad9": dict(n_nodes=9, n_corners=4, family="quad", order=2,
                  edges=[(0, 1, 4), (1, 2, 5), (2, 3, 6), (3, 0, 7)], gauss=("tensor", 3)),
    "tri3": dict(n_nodes=3, n_corners=3, family="tri", order=1,
                 edges=[(0, 1), (1, 2), (2, 0)], gauss=("triangle", 1)),
    "tri6": dict(n_nodes=6, n_corners=3, family="tri", order=2,
                 edges=[(0, 1, 3), (1, 2, 4), (2, 0, 5)], gauss=("triangle", 4)),
}


def element_names():
    return list(ELEMENT_LIBRARY)


def get_element(name):
    if name not in ELEMENT_LIBRARY:
        raise ValueError(f"Unknown element type '{name}'. Choose one of {element_names()}.")
    return ELEMENT_LIBRARY[name]


# ---------------------------------------------------------------------------------------------
# quadrature
# ---------------------------------------------------------------------------------------------
# Published degree-4 six-point rule on the triangle (two orbits (a, a, 1 - 2a)); weights sum to 1 on the
# unit-area triangle.  These are the same 15-digit constants the reference uses
# (gauss_quadratures.py:136-142), so that Tri6 Gauss data agree bit for bit.
_TRI6_A = (0.445948490915965, 0.091576213509771)
_TRI6_W = (0.223381589678011, 0.109951743655322)


# Quadrature rules depend on (rule, dtype, device) only: each is built once and shared, so a serving thread
# does not rebuild them (and copy them to the device) for every request.  The returned tensors are shared:
# callers must not modify them.  A CUDA rule is cached after its blocking host-to-device copy has completed,
# so threads on other streams may read it at once.
_QUADRATURE = {}


def _device_key(device):
    d = torch.device(device)
    if d.type == "cuda" and d.index is None:
        d = torch.device("cuda", torch.cuda.current_device())
    return str(d)


def _cached_rule(key, build):
    rule = _QUADRATURE.get(key)
    if rule is None:
        rule = _QUADRATURE.setdefault(key, build())
    return rule


def gauss_1d(n, dtype=torch.float64, device="cpu"):
    """n-point Gauss-Legendre rule on [-1, 1] (points, weights); cached and shared (do not modify)."""
    def build():
        x, w = np.polynomial.legendre.leggauss(n)
        return torch.tensor(x, dtype=dtype, device=device), torch.tensor(w, dtype=dtype, device=device)
    return _cached_rule(("gauss_1d", n, dtype, _device_key(device)), build)


def gauss_square(n, dtype=torch.float64, device="cpu"):
    """Tensor rule on [-1, 1]^2, eta-major / xi-minor ordering (point k = (x[k % n], x[k // n]))."""
    x, w = gauss_1d(n, dtype, device)
    xi = x.repeat(n)
    eta = x.repeat_interleave(n)
    return torch.stack([xi, eta], dim=1), (w[:, None] * w[None, :]).reshape(-1)


def gauss_triangle(degree, dtype=torch.float64, device="cpu"):
    """Rules on the reference triangle used by the element library (degree 1 and 4)."""
    if degree <= 1:
        pts, wts = [[1.0 / 3.0, 1.0 / 3.0]], [0.5]
    elif degree <= 4:
        pts, wts = [], []
        for a, w in zip(_TRI6_A, _TRI6_W):
            b = 1.0 - 2.0 * a
            pts += [[a, a], [b, a], [a, b]]
            wts += [0.5 * w] * 3
    else:
        raise ValueError("only the degree-1 and degree-4 triangle rules of the element library are provided")
    return torch.tensor(pts, dtype=dtype, device=device), torch.tensor(wts, dtype=dtype, device=device)


def default_rule(name, points):
    """True when ``points`` is the (shared) point tensor of this library's default rule of element ``name``."""
    rule = _QUADRATURE.get(("element", name, points.dtype, _device_key(points.device)))
    return rule is not None and rule[0] is points


_RULE_GRADIENTS = {}


def quadrature_gradients(name, points):
    """
    shape_gradients of element ``name`` at the points (n_q, 2).  For the default rule's shared point tensor
    the result is computed once and shared as well (do not modify); a CUDA result is cached after its
    stream has finished computing it, so threads on other streams may read it at once.
    """
    key = (name, id(points))
    hit = _RULE_GRADIENTS.get(key)
    if hit is not None and hit[0] is points:
        return hit[1]
    g = shape_gradients(name, points[:, 0], points[:, 1])
    if default_rule(name, points):
        if g.is_cuda:
            torch.cuda.current_stream(g.device).synchronize()
        _RULE_GRADIENTS[key] = (points, g)
    return g


def element_quadrature(name, dtype=torch.float64, device="cpu"):
    """Default Gauss rule (points (n_q, 2), weights (n_q,)) of an element type; cached and shared (do not
    modify)."""
    kind, n = get_element(name)["gauss"]
    return _cached_rule(("element", name, dtype, _device_key(device)),
                        lambda: gauss_square(n, dtype, device) if kind == "tensor" else gauss_triangle(n, dtype, device))


# ---------------------------------------------------------------------------------------------
# shape functions (values) and reference gradients, vectorised over points
# ---------------------------------------------------------------------------------------------
def _lagrange3(s):
    """Quadratic Lagrange polynomials at s = -1, 0, +1 and their derivatives."""
    L = (0.5 * s * (s - 1.0), 1.0 - s * s, 0.5 * s * (s + 1.0))
    dL = (s - 0.5, -2.0 * s, s + 0.5)
    return L, dL


# (xi index, eta index) of every Q9 node in the 3x3 Lagrange grid, local ordering of the library
_Q9_IJ = [(0, 0), (2, 0), (2, 2), (0, 2), (1, 0), (2, 1), (1, 2), (0, 1), (1, 1)]
_Q_CORNERS = [(-1.0, -1.0), (1.0, -1.0), (1.0, 1.0), (-1.0, 1.0)]


def shape_values(name, xi, eta):
    """N_a(xi, eta) for every node a; xi, eta tensors of equal shape -> (..., nen)."""
    if name == "quad4":
        return torch.stack([0.25 * (1 + a * xi) * (1 + b * eta) for a, b in _Q_CORNERS], dim=-1)
    if name == "quad9":
        Lx, _ = _lagrange3(xi)
        Ly, _ = _lagrange3(eta)
        return torch.stack([Lx[i] * Ly[j] for i, j in _Q9_IJ], dim=-1)
    if name == "quad8":
        corners = [0.25 * (1 + a * xi) * (1 + b * eta) * (a * xi + b * eta - 1) for a, b in _Q_CORNERS]
        mids = [0.5 * (1 - xi * xi) * (1 - eta), 0.5 * (1 + xi) * (1 - eta * eta),
                0.5 * (1 - xi * xi) * (1 + eta), 0.5 * (1 - xi) * (1 - eta * eta)]
        return torch.stack(corners + mids, dim=-1)
    l1, l2, l3 = 1.0 - xi - eta, xi, eta
    if name == "tri3":
        return torch.stack([l1, l2, l3], dim=-1)
    if name == "tri6":
        return torch.stack([l1 * (2 * l1 - 1), l2 * (2 * l2 - 1), l3 * (2 * l3 - 1),
                            4 * l1 * l2, 4 * l2 * l3, 4 * l3 * l1], dim=-1)
    raise ValueError(f"Unknown element type '{name}'")


def shape_gradients(name, xi, eta):
    """dN_a/d(xi, eta) in closed form; xi, eta tensors of equal shape -> (..., nen, 2)."""
    if name == "quad4":
        g = [(0.25 * a * (1 + b * eta), 0.25 * b * (1 + a * xi)) for a, b in _Q_CORNERS]
    elif name == "quad9":
        Lx, dLx = _lagrange3(xi)
        Ly, dLy = _lagrange3(eta)
        g = [(dLx[i] * Ly[j], Lx[i] * dLy[j]) for i, j in _Q9_IJ]
    elif name == "quad8":
        g = [(0.25 * a * (1 + b * eta) * (2 * a * xi + b * eta), 0.25 * b * (1 + a * xi) * (a * xi + 2 * b * eta))
             for a, b in _Q_CORNERS]
        g += [(-xi * (1 - eta), -0.5 * (1 - xi * xi)), (0.5 * (1 - eta * eta), -eta * (1 + xi)),
              (-xi * (1 + eta), 0.5 * (1 - xi * xi)), (-0.5 * (1 - eta * eta), -eta * (1 - xi))]
    elif name in ("tri3", "tri6"):
        one, zero = torch.ones_like(xi), torch.zeros_like(xi)
        dl = [(-one, -one), (one, zero), (zero, one)]
        if name == "tri3":
            g = dl
        else:
            lam = [1.0 - xi - eta, xi, eta]
            g = [((4 * lam[k] - 1) * dl[k][0], (4 * lam[k] - 1) * dl[k][1]) for k in range(3)]
            for i, j in ((0, 1), (1, 2), (2, 0)):
                g.append((4 * (lam[j] * dl[i][0] + lam[i] * dl[j][0]), 4 * (lam[j] * dl[i][1] + lam[i] * dl[j][1])))
    else:
        raise ValueError(f"Unknown element type '{name}'")
    return torch.stack([torch.stack([gx, gy], dim=-1) for gx, gy in g], dim=-2)


def make_shape_fn(name):
    """Callable (xi, eta) -> (nen,) like the reference's params["shape_fn"]."""
    get_element(name)

    def shape_fn(xi, eta):
        return shape_values(name, torch.as_tensor(xi), torch.as_tensor(eta))
    shape_fn.element_type = name
    return shape_fn


# ---------------------------------------------------------------------------------------------
# edges (1D) for traction loads
# ---------------------------------------------------------------------------------------------
def edge_shape(order, s):
    """1D edge shape functions and derivatives: ends first, then the mid node (quadratic)."""
    if order == 1:
        N = torch.stack([0.5 * (1 - s), 0.5 * (1 + s)], dim=-1)
        dN = torch.stack([torch.full_like(s, -0.5), torch.full_like(s, 0.5)], dim=-1)
    else:
        N = torch.stack([0.5 * s * (s - 1), 0.5 * s * (s + 1), 1 - s * s], dim=-1)
        dN = torch.stack([s - 0.5, s + 0.5, -2 * s], dim=-1)
    return N, dN


_EDGE_SHAPES = {}


def edge_shape_at_rule(order, s):
    """edge_shape(order, s); for a shared Gauss rule's points (gauss_1d) the result is computed once and shared
    as well (do not modify), after its stream has finished computing it."""
    key = (order, id(s))
    hit = _EDGE_SHAPES.get(key)
    if hit is not None and hit[0] is s:
        return hit[1]
    out = edge_shape(order, s)
    if any(rule[0] is s for k, rule in list(_QUADRATURE.items()) if k[0] == "gauss_1d"):
        if s.is_cuda:
            torch.cuda.current_stream(s.device).synchronize()
        _EDGE_SHAPES[key] = (s, out)
    return out


def reference_node_coordinates(name, dtype=torch.float64):
    coords = {
        "quad4": [(-1, -1), (1, -1), (1, 1), (-1, 1)],
        "quad8": [(-1, -1), (1, -1), (1, 1), (-1, 1), (0, -1), (1, 0), (0, 1), (-1, 0)],
        "quad9": [(-1, -1), (1, -1), (1, 1), (-1, 1), (0, -1), (1, 0), (0, 1), (-1, 0), (0, 0)],
        "tri3": [(0, 0), (1, 0), (0, 1)],
        "tri6": [(0, 0), (1, 0), (0, 1), (0.5, 0), (0.5, 0.5), (0, 0.5)],
    }[name]
    return torch.tensor(coords, dtype=dtype)


def n_quadrature_points(name):
    kind, n = get_element(name)["gauss"]
    return n * n if kind == "tensor" else (1 if n <= 1 else 6)
