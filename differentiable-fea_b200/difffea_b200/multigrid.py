"""
Geometric multigrid preconditioner for structured quadrilateral meshes (preconditioner="multigrid").

The reference's preconditioners are Jacobi, nodal block-Jacobi and an incomplete LU on the CPU
(operators.py:477-710); it names a scalable preconditioner as its main open item (docs/ROADMAP.md:11).
This module builds one for the meshes whose cells form a logical grid (every rectangle of the
structured mesher, Q4 or Q9, and the mapped quarter plate):

    level 0     the finite-element mesh and its operator A = M K M + (I - M) (stored moduli, kernel (b))
    level 1     a Q4 grid on the element corners (Q9: the element grid itself; Q4: every other line)
    level l+1   every other grid line of level l (a last cell one line wide when the count is odd),
                down to at most 128 nodes, where the operator is inverted densely

Coarse operators are Galerkin products assembled element by element on the device (K_C = sum (B P~)^T
C (B P~) from the fine moduli, then sum P^T K P), P~ the bilinear interpolation with fixed fine DOFs
zeroed, so every coarse operator is P~^T A P~ exactly (to rounding) and SPD.  Smoothing is Chebyshev
with the Jacobi diagonal of each level on [lambda_max / 10, 1.1 lambda_max], lambda_max of D^-1 A from
10 Lanczos steps per level and linearisation (the coefficients of Jacobi-preconditioned CG, all levels in
lockstep with their scalars on the device, one host read): power iteration converges too slowly for the
dense top of this spectrum (26 % low after 10 steps on a 256 x 64 Q4 cantilever, measured, which made the
smoother amplify the highest modes), Lanczos is within 1 % after 10.  The same polynomial runs before and
after the coarse correction, so the V-cycle is a symmetric positive definite preconditioner for PCG.
"""
import ctypes
import math

import torch

from difffea_b200 import _lib
from difffea_b200.cuda_mesh import ptr, stream_handle

COARSEST_NODES = 128          # levels are coarsened until a level has at most this many nodes
CHEB_DEGREE = 2
CHEB_RATIO = 10.0             # smoothing interval [lambda_max / ratio, 1.1 lambda_max]
LANCZOS_STEPS = 10


# ---------------------------------------------------------------------------------------------
# the grid behind a structured mesh
# ---------------------------------------------------------------------------------------------
def _grid_conn(ids, ncx, ncy, span):
    """Connectivity of an ncx x ncy cell grid over node ids (grid of span*ncx+1 x span*ncy+1 nodes)."""
    if span == 1:
        c = [ids[:ncx, :ncy], ids[1:ncx + 1, :ncy], ids[1:ncx + 1, 1:ncy + 1], ids[:ncx, 1:ncy + 1]]
        return torch.stack([t.reshape(-1) for t in c], dim=1)
    offs = [(0, 0), (2, 0), (2, 2), (0, 2), (1, 0), (2, 1), (1, 2), (0, 1), (1, 1)]
    return torch.stack([ids[di:di + 2 * ncx:2, dj:dj + 2 * ncy:2].reshape(-1) for di, dj in offs], dim=1)


def structured_grid(conn, n_nodes):
    """
    The logical grid of a structured Q4 / Q9 mesh, or None: tries every cell count ncx x ncy = n_el
    with the node numbering of the rectangle mesher (grid node (i, j) = i (gy + 1) + j) and of the
    quarter-plate mesher (i + j (gx + 1)), and accepts one whose connectivity matches exactly.
    Returns dict(span, ncx, ncy, gx, gy, gnode (grid -> FE node), node_ij (FE node -> grid)).
    """
    n_el, nen = conn.shape
    span = {4: 1, 9: 2}.get(nen)
    if span is None or n_el == 0:
        return None
    dev = conn.device
    for ncx in range(1, n_el + 1):
        if n_el % ncx:
            continue
        ncy = n_el // ncx
        gx, gy = span * ncx, span * ncy
        if (gx + 1) * (gy + 1) != n_nodes:
            continue
        lex = torch.arange((gx + 1) * (gy + 1), device=dev)
        for ids in (lex.reshape(gx + 1, gy + 1), lex.reshape(gy + 1, gx + 1).t()):
            if torch.equal(_grid_conn(ids, ncx, ncy, span), conn):
                gnode = ids.reshape(-1).to(torch.int32).contiguous()
                node_ij = torch.empty(n_nodes, 2, dtype=torch.int32, device=dev)
                ii = torch.arange(gx + 1, device=dev)[:, None].expand(gx + 1, gy + 1).reshape(-1)
                jj = torch.arange(gy + 1, device=dev)[None, :].expand(gx + 1, gy + 1).reshape(-1)
                node_ij[gnode.long(), 0] = ii.to(torch.int32)
                node_ij[gnode.long(), 1] = jj.to(torch.int32)
                return dict(span=span, ncx=ncx, ncy=ncy, gx=gx, gy=gy, gnode=gnode, node_ij=node_ij.contiguous())
    return None


# ---------------------------------------------------------------------------------------------
# hierarchy
# ---------------------------------------------------------------------------------------------
class _Level:
    def __init__(self, gx, gy, finer=None, device="cuda"):
        self.gx, self.gy = gx, gy
        self.n_nodes = (gx + 1) * (gy + 1)
        self.n = 2 * self.n_nodes
        i32 = dict(dtype=torch.int32, device=device)
        self.keep = []
        self.grid = _lib.MgGrid()
        self.grid.gx, self.grid.gy = gx, gy
        if finer is not None:
            fgx, fgy = finer.gx, finer.gy
            lx = torch.tensor([min(2 * i, fgx) for i in range(gx + 1)], **i32)
            ly = torch.tensor([min(2 * j, fgy) for j in range(gy + 1)], **i32)
            cx = torch.tensor([min(i // 2, gx - 1) for i in range(fgx + 1)], **i32)
            cy = torch.tensor([min(j // 2, gy - 1) for j in range(fgy + 1)], **i32)
            self.K = torch.empty(64 * gx * gy, dtype=torch.float64, device=device)
            self.fix = torch.empty(self.n_nodes, dtype=torch.uint8, device=device)
            self.keep += [lx, ly, cx, cy]
            for name, t in (("line_x", lx), ("line_y", ly), ("cell_x", cx), ("cell_y", cy), ("K", self.K),
                            ("fix", self.fix)):
                setattr(self.grid, name, t.data_ptr())
        f64 = dict(dtype=torch.float64, device=device)
        self.diag = torch.empty(self.n, **f64)
        self.b, self.x, self.r = (torch.empty(self.n, **f64) for _ in range(3))
        self.d, self.q = torch.empty(self.n, **f64), torch.empty(self.n, **f64)
        self.lam = 1.0

    @property
    def ref(self):
        return ctypes.byref(self.grid)


def _coarser(g):
    return max(1, (g + 1) // 2)


def _ritz_max(hist):
    """Largest eigenvalue of the Lanczos tridiagonal matrix of CG coefficients (alpha_k, beta_k) pairs, over the
    prefix before any breakdown (alpha <= 0, beta < 0 or not finite)."""
    import numpy as np
    a, b = hist[0::2], hist[1::2]
    m = 0
    while m < len(a) and np.isfinite(a[m]) and a[m] > 0 and np.isfinite(b[m]) and b[m] >= 0:
        m += 1
    if m == 0:
        return 2.5
    T = np.zeros((m, m))
    for k in range(m):
        T[k, k] = 1.0 / a[k] + (b[k - 1] / a[k - 1] if k > 0 else 0.0)
        if k + 1 < m:
            T[k, k + 1] = T[k + 1, k] = math.sqrt(b[k]) / a[k]
    return float(np.linalg.eigvalsh(T).max())


class Multigrid:
    """V-cycle preconditioner r -> z of one structured mesh; ``setup`` at every linearisation."""

    def __init__(self, mesh, params, degree=CHEB_DEGREE, ratio=CHEB_RATIO, lanczos_steps=LANCZOS_STEPS):
        g = structured_grid(params["conn"].to(mesh.device), mesh.n_nodes)
        if g is None:
            raise ValueError("preconditioner='multigrid' needs a structured Q4 or Q9 mesh (a logical grid of cells)")
        self.mesh, self.g = mesh, g
        self.degree, self.ratio, self.lanczos_steps = degree, ratio, lanczos_steps
        dev = mesh.device
        inv_perm = torch.empty_like(mesh.perm)
        inv_perm[mesh.perm] = torch.arange(mesh.perm.numel(), device=dev)
        self.cell_slot = inv_perm.to(torch.int32).contiguous()      # cells are numbered like the elements
        self.levels = [_Level(g["gx"], g["gy"], None, dev)]
        while True:
            f = self.levels[-1]
            if len(self.levels) > 1 and (f.n_nodes <= COARSEST_NODES or (f.gx == 1 and f.gy == 1)):
                break
            self.levels.append(_Level(_coarser(f.gx), _coarser(f.gy), f, dev))
        last = self.levels[-1]
        if last.n > int(_lib.load().dfea_mg_dense_max()):
            raise ValueError("multigrid: the coarsest level is too large for the dense solve")
        self.Ainv = torch.empty(last.n * last.n, dtype=torch.float64, device=dev)
        self.dense_work = torch.empty_like(self.Ainv)
        self.dots = torch.zeros(2, dtype=torch.float64, device=dev)
        n_s = len(self.levels) - 1
        self.lscal = torch.zeros(n_s, 4, dtype=torch.float64, device=dev)
        self.lhist = torch.zeros(n_s, 2 * lanczos_steps, dtype=torch.float64, device=dev)
        self._start = [torch.sin(torch.arange(1, lv.n + 1, dtype=torch.float64, device=dev)) for lv in self.levels]
        self.C, self.code = None, None

    # -- operators -------------------------------------------------------------------------------
    def _apply(self, l, v, y):
        if l == 0:
            _lib.call("dfea_tangent_apply", self.mesh.view_ref, ptr(self.C), self.code, ptr(v), ptr(y), _lib.DFEA_F64,
                      stream_handle())
        else:
            _lib.call("dfea_mg_apply", self.levels[l].ref, ptr(v), ptr(y), stream_handle())

    def _transfer_args(self, l):
        f, c = self.levels[l], self.levels[l + 1]
        if l == 0:
            return f.ref, c.ref, ptr(self.g["gnode"]), ptr(self.mesh.node_fix)
        return f.ref, c.ref, ptr(None), ptr(f.fix)

    # -- set-up at a linearisation ---------------------------------------------------------------
    def setup(self, C, moduli_code, diag):
        """Coarse operators from the fine moduli C (DFEA_F64 / DFEA_F32 / DFEA_F32REF) and the Jacobi diagonal."""
        self.C, self.code = C, moduli_code
        lv0 = self.levels[0]
        lv0.diag.copy_(diag)
        s = stream_handle()
        for l in range(1, len(self.levels)):
            fr, cr, gn, ffix = self._transfer_args(l - 1)
            _lib.call("dfea_mg_restrict", fr, cr, gn, ffix, ptr(None), ptr(None), ptr(self.levels[l].fix), s)
            if l == 1:
                _lib.call("dfea_mg_galerkin_fe", self.mesh.view_ref, ptr(C), moduli_code, ptr(self.g["node_ij"]),
                          ptr(self.cell_slot), self.g["span"], lv0.ref, self.levels[1].ref, s)
            else:
                _lib.call("dfea_mg_galerkin", self.levels[l - 1].ref, self.levels[l].ref, s)
            _lib.call("dfea_mg_diag", self.levels[l].ref, ptr(self.levels[l].diag), s)
        last = self.levels[-1]
        _lib.call("dfea_mg_dense_inverse", last.ref, ptr(self.dense_work), ptr(self.Ainv), s)
        # lambda_max(D^-1 A) per smoothed level by Lanczos: r = start, z = r / D, p = z (p in x, z in d)
        smoothed = self.levels[:-1]
        for l, lv in enumerate(smoothed):
            lv.r.copy_(self._start[l])
            _lib.call("dfea_mg_cheb_start", lv.n, ptr(lv.r), ptr(lv.diag), 1.0, ptr(lv.d), s)
            lv.x.copy_(lv.d)
            _lib.call("dfea_mg_dot", lv.n, ptr(lv.r), ptr(lv.d), ptr(self.lscal[l, 1:]), s)
        for k in range(self.lanczos_steps):
            for l, lv in enumerate(smoothed):
                self._apply(l, lv.x, lv.q)
                _lib.call("dfea_mg_lanczos_step", lv.n, ptr(lv.x), ptr(lv.q), ptr(lv.r), ptr(lv.d), ptr(lv.diag),
                          ptr(self.lscal[l]), ptr(self.lhist[l]), k, s)
        hist = self.lhist.cpu().numpy()
        for l, lv in enumerate(smoothed):
            lv.lam = _ritz_max(hist[l])

    # -- the cycle --------------------------------------------------------------------------------
    def _cheb(self, l, x, r):
        lv, s = self.levels[l], stream_handle()
        hi = 1.1 * lv.lam
        lo = hi / self.ratio
        theta, delta = 0.5 * (hi + lo), 0.5 * (hi - lo)
        sigma = theta / delta
        rho = 1.0 / sigma
        _lib.call("dfea_mg_cheb_start", lv.n, ptr(r), ptr(lv.diag), 1.0 / theta, ptr(lv.d), s)
        for k in range(1, self.degree + 1):
            self._apply(l, lv.d, lv.q)
            last = k == self.degree
            c1 = c2 = 0.0
            if not last:
                rho_new = 1.0 / (2.0 * sigma - rho)
                c1, c2 = rho_new * rho, 2.0 * rho_new / delta
                rho = rho_new
            _lib.call("dfea_mg_cheb_step", lv.n, ptr(x), ptr(r), ptr(lv.d), ptr(lv.q), ptr(lv.diag), c1, c2,
                      1 if last else 0, s)

    def _vcycle(self, l, b, x):
        s = stream_handle()
        lv = self.levels[l]
        if l == len(self.levels) - 1:
            _lib.call("dfea_mg_dense_solve", lv.n, ptr(self.Ainv), ptr(b), ptr(x), s)
            return
        lv.r.copy_(b)
        x.zero_()
        self._cheb(l, x, lv.r)
        c = self.levels[l + 1]
        fr, cr, gn, ffix = self._transfer_args(l)
        _lib.call("dfea_mg_restrict", fr, cr, gn, ffix, ptr(lv.r), ptr(c.b), ptr(None), s)
        self._vcycle(l + 1, c.b, c.x)
        _lib.call("dfea_mg_prolong_add", fr, cr, gn, ffix, ptr(c.x), ptr(x), s)
        self._apply(l, x, lv.q)
        _lib.call("dfea_add_scaled", lv.n, ptr(b), -1.0, ptr(lv.q), ptr(lv.r), s)
        self._cheb(l, x, lv.r)

    def apply(self, r, z):
        """z = M^-1 r (one V-cycle); r and z are (2N,) float64 device vectors."""
        self._vcycle(0, r, z)
        return z

    def __call__(self, r):
        z = torch.empty_like(r)
        return self.apply(r.contiguous(), z)


def mg_pcg(apply_A, mg, b, x, rtol, max_iter, work):
    """
    PCG (Saad, Alg. 9.1) for A x = b with the V-cycle as preconditioner, x0 = 0, on device vectors; the
    host reads three scalars per iteration (p.Ap, ||r||^2, r.z).  Returns (iterations, status) with the
    statuses of the device PCG: "converged", "max_iter", "negative_curvature", "zero_rhs".
    ``work``: a (4, 2N) float64 buffer (r, z, p, q).
    """
    n, s = b.numel(), stream_handle()
    r, z, p, q = work[0], work[1], work[2], work[3]
    dots = mg.dots

    def dot(u, v):
        _lib.call("dfea_mg_dot", n, ptr(u), ptr(v), ptr(dots), s)
        return float(dots[0])

    x.zero_()
    r.copy_(b)
    nb2 = dot(b, b)
    if nb2 == 0.0:
        return 0, _lib.PCG_STATUS[4]
    tol2 = rtol * rtol * nb2
    mg.apply(r, z)
    p.copy_(z)
    rz = dot(r, z)
    for k in range(max_iter):
        apply_A(p, q)
        curv = dot(p, q)
        if not curv > 0.0:
            if k == 0:
                x.copy_(z)
            return k, _lib.PCG_STATUS[3]
        alpha = rz / curv
        _lib.call("dfea_axpy", n, alpha, ptr(p), ptr(x), s)
        _lib.call("dfea_axpy", n, -alpha, ptr(q), ptr(r), s)
        if dot(r, r) <= tol2:
            return k + 1, _lib.PCG_STATUS[1]
        mg.apply(r, z)
        rz_new = dot(r, z)
        _lib.call("dfea_add_scaled", n, ptr(z), rz_new / rz, ptr(p), ptr(p), s)
        rz = rz_new
    return max_iter, _lib.PCG_STATUS[2]
