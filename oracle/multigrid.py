"""
CPU restatement of the geometric multigrid V-cycle (test infrastructure, like the rest of oracle/).

The reference has no multigrid (its preconditioners are Jacobi, block-Jacobi and ILU, operators.py:477-710;
a scalable one is its open item, docs/ROADMAP.md:11), so this module restates the algorithm the CUDA path
implements, with dense matrices, for small structured rectangle meshes (grid node (i, j) = FE node
i (gy + 1) + j, the rectangle mesher's numbering):

    A_0 = M K M + (I - M) assembled column by column from the oracle's tangent product
    P_l  bilinear interpolation from level l+1 (every other grid line, a last cell one line wide when the
         count is odd) to level l, P~_l = M_l P_l
    M_{l+1}: a coarse DOF is free when any fine DOF it interpolates to is free
    A_{l+1} = P~_l^T A_l P~_l + (I - M_{l+1})
    smoothing: Chebyshev iteration with the Jacobi diagonal on [lambda/10, 1.1 lambda]... see vcycle()
"""
import math

import torch

from oracle.reference_path import F64, make_operator

COARSEST_NODES = 48


def _coarser(g):
    return max(1, (g + 1) // 2)


def _interp_1d(gf, gc):
    """(gf+1, gc+1) weights of coarse lines (at fine lines min(2I, gf)) at every fine line."""
    lines = [min(2 * i, gf) for i in range(gc + 1)]
    W = torch.zeros(gf + 1, gc + 1, dtype=F64)
    for i in range(gf + 1):
        c = min(i // 2, gc - 1)                    # the coarse cell holding fine line i
        a, b = lines[c], lines[c + 1]
        W[i, c] = (b - i) / (b - a)
        W[i, c + 1] = (i - a) / (b - a)
    return W


def hierarchy(A0, gx, gy, fixed0, diag0=None, node_ij=None):
    """
    Levels [(A, P~ to the finer level, fixed)] of the V-cycle; fixed0: (2N,) bool.  node_ij: (N, 2) grid
    position of every FE node (default: all grid nodes, numbered i (gy + 1) + j) -- level 0's interpolation
    is evaluated at those positions, so meshes whose nodes are a subset of the grid (Q8) work alike.
    """
    levels = [dict(A=A0, fixed=fixed0, gx=gx, gy=gy, diag=diag0 if diag0 is not None else torch.diagonal(A0).clone())]
    while True:
        f = levels[-1]
        nn = (f["gx"] + 1) * (f["gy"] + 1)
        if len(levels) > 1 and (nn <= COARSEST_NODES or (f["gx"] == 1 and f["gy"] == 1)):
            break
        cgx, cgy = _coarser(f["gx"]), _coarser(f["gy"])
        Wn = torch.kron(_interp_1d(f["gx"], cgx), _interp_1d(f["gy"], cgy))          # nodes
        if len(levels) == 1 and node_ij is not None:
            Wn = Wn[node_ij[:, 0] * (f["gy"] + 1) + node_ij[:, 1]]
        P = torch.kron(Wn, torch.eye(2, dtype=F64))                                    # DOFs (2 node + comp)
        Pt = P * (~f["fixed"]).to(F64)[:, None]
        fixed_c = (Pt.abs().sum(0) == 0)
        K = f["A"] * (~f["fixed"]).to(F64)[:, None] * (~f["fixed"]).to(F64)[None, :]
        A = Pt.T @ K @ Pt + torch.diag(fixed_c.to(F64))
        levels[-1]["P"] = Pt
        levels.append(dict(A=A, fixed=fixed_c, gx=cgx, gy=cgy, diag=torch.diagonal(A).clone()))
    return levels


def lambda_max(A, diag, steps=10):
    """Lanczos estimate of lambda_max(D^-1 A): the tridiagonal matrix of `steps` Jacobi-CG coefficients from
    b = sin(1..n) (Saad, Iterative Methods, section 6.7)."""
    r = torch.sin(torch.arange(1, A.shape[0] + 1, dtype=F64))
    z = r / diag
    p = z.clone()
    rz = float(r @ z)
    a, b = [], []
    for _ in range(steps):
        q = A @ p
        alpha = rz / float(p @ q)
        r = r - alpha * q
        z = r / diag
        rz_new = float(r @ z)
        beta = rz_new / rz
        p = z + beta * p
        rz = rz_new
        a.append(alpha)
        b.append(beta)
        if not (math.isfinite(alpha) and alpha > 0 and math.isfinite(beta) and beta >= 0):
            a.pop()
            b.pop()
            break
    m = len(a)
    if m == 0:
        return 2.5
    T = torch.zeros(m, m, dtype=F64)
    for k in range(m):
        T[k, k] = 1.0 / a[k] + (b[k - 1] / a[k - 1] if k > 0 else 0.0)
        if k + 1 < m:
            T[k, k + 1] = T[k + 1, k] = math.sqrt(b[k]) / a[k]
    return float(torch.linalg.eigvalsh(T).max())


def chebyshev(A, diag, lam, x, r, degree=2, ratio=10.0):
    """degree steps of the Jacobi-preconditioned Chebyshev iteration (Saad, Alg. 12.1); updates x, r."""
    hi = 1.1 * lam
    lo = hi / ratio
    theta, delta = 0.5 * (hi + lo), 0.5 * (hi - lo)
    sigma = theta / delta
    rho = 1.0 / sigma
    d = r / diag / theta
    for k in range(1, degree + 1):
        x = x + d
        r = r - A @ d
        if k < degree:
            rho_new = 1.0 / (2.0 * sigma - rho)
            d = rho_new * rho * d + (2.0 * rho_new / delta) * r / diag
            rho = rho_new
    return x, r


def vcycle(levels, b, l=0, lams=None):
    lv = levels[l]
    if l == len(levels) - 1:
        return torch.linalg.solve(lv["A"], b)
    lam = lams[l]
    x, r = chebyshev(lv["A"], lv["diag"], lam, torch.zeros_like(b), b.clone())
    e = vcycle(levels, lv["P"].T @ r, l + 1, lams)
    x = x + lv["P"] @ e
    x, _ = chebyshev(lv["A"], lv["diag"], lam, x, b - lv["A"] @ x)
    return x


def preconditioner(u, theta, P, gx, gy, diag0=None, node_ij=None):
    """The V-cycle r -> z at (u, theta) for a structured mesh of gx x gy node-grid cells."""
    A_fn = make_operator("qp", u, theta, P)
    n = u.numel()
    A0 = torch.stack([A_fn(torch.eye(n, dtype=F64)[i]) for i in range(n)], dim=1)
    levels = hierarchy(A0, gx, gy, P["fixed"].clone(), diag0, node_ij)
    lams = [lambda_max(lv["A"], lv["diag"]) for lv in levels[:-1]]
    return (lambda r: vcycle(levels, r, 0, lams)), levels, lams
