"""
Geometric multigrid preconditioner for structured quadrilateral meshes (preconditioner="multigrid").

The reference's preconditioners are Jacobi, nodal block-Jacobi and an incomplete LU on the CPU
(operators.py:477-710); it names a scalable preconditioner as its main open item (docs/ROADMAP.md:11).
This module builds one for the meshes whose cells form a logical grid (every rectangle of the
structured mesher, any element type, and the mapped quarter plate):

    level 0     the finite-element mesh and its operator A = M K M + (I - M) (stored moduli, kernel (b))
    level 1     a Q4 grid on the element corners (Q9 / Q8 / Tri6: the element grid; Q4 / Tri3: every other line)
    level l+1   every other grid line of level l (a last cell one line wide when the count is odd),
                down to at most 48 nodes, where the operator is inverted densely

Coarse operators are Galerkin products assembled element by element on the device (K_C = sum (B P~)^T
C (B P~) from the fine moduli, then sum P^T K P), P~ the bilinear interpolation with fixed fine DOFs
zeroed, so every coarse operator is P~^T A P~ exactly (to rounding) and SPD.  Smoothing is Chebyshev
with the Jacobi diagonal of each level on [lambda / 10, lambda], lambda = 1.1 x the lambda_max of D^-1 A from
10 Lanczos steps per level and linearisation (the coefficients of Jacobi-preconditioned CG, all levels in
lockstep with their scalars on the device, one host read): power iteration converges too slowly for the
dense top of this spectrum (26 % low after 10 steps on a 256 x 64 Q4 cantilever, measured, which made the
smoother amplify the highest modes), Lanczos is within 1 % after 10.  The same polynomial runs before and
after the coarse correction, so the V-cycle is a symmetric positive definite preconditioner for PCG.
Set-up, cycle and the PCG loop run in the library's C++ driver (dfea_mg_setup / dfea_mg_vcycle /
dfea_mg_pcg); this module builds the grid description and owns the buffers.
"""
import ctypes
import math

import torch

from difffea_b200 import _lib, ops

COARSEST_NODES = 48           # levels are coarsened until a level has at most this many nodes (96 DOFs: the
                              # dense Gauss-Jordan of the coarsest operator then runs in shared memory)
CHEB_DEGREE = 2
CHEB_RATIO = 10.0             # smoothing interval [lambda_max / ratio, 1.1 lambda_max]
LANCZOS_STEPS = 10


# ---------------------------------------------------------------------------------------------
# the grid behind a structured mesh
# ---------------------------------------------------------------------------------------------
# per element type (nodes per element): grid cells spanned by an element, elements per cell
_LAYOUT = {4: (1, 1), 9: (2, 1), 8: (2, 1), 3: (1, 2), 6: (2, 2)}


def _grid_conn(ids, ncx, ncy, nen):
    """
    Connectivity of an ncx x ncy cell grid over the grid node ids, in the element library's local order:
    Q4 / Q9 / Q8 one element per cell, Tri3 / Tri6 the lower-left triangles of all cells, then the
    upper-right ones.
    """
    if nen in (4, 3):
        c = [ids[:ncx, :ncy], ids[1:ncx + 1, :ncy], ids[1:ncx + 1, 1:ncy + 1], ids[:ncx, 1:ncy + 1]]
        q4 = torch.stack([t.reshape(-1) for t in c], dim=1)
        return q4 if nen == 4 else torch.cat([q4[:, [0, 1, 3]], q4[:, [1, 2, 3]]], dim=0)
    offs = [(0, 0), (2, 0), (2, 2), (0, 2), (1, 0), (2, 1), (1, 2), (0, 1), (1, 1)]
    q9 = torch.stack([ids[di:di + 2 * ncx:2, dj:dj + 2 * ncy:2].reshape(-1) for di, dj in offs], dim=1)
    if nen == 9:
        return q9
    if nen == 8:
        return q9[:, :8]
    return torch.cat([q9[:, [0, 1, 3, 4, 8, 7]], q9[:, [1, 2, 3, 5, 6, 8]]], dim=0)


def _candidates(n_cells, n_nodes, span, q8):
    """(ncx, ncy) with ncx ncy = n_cells and the node count of the grid: N = span^2 cells + span (ncx + ncy)
    + 1, minus the cell centres for Q8; ncx and ncy are the roots of t^2 - (ncx + ncy) t + cells."""
    rest = n_nodes - 1 - (span * span - (1 if q8 else 0)) * n_cells
    if rest <= 0 or rest % span:
        return []
    ssum = rest // span
    disc = ssum * ssum - 4 * n_cells
    if disc < 0:
        return []
    root = math.isqrt(disc)
    if root * root != disc or (ssum + root) % 2:
        return []
    out = []
    for ncx in sorted({(ssum - root) // 2, (ssum + root) // 2}):
        if ncx >= 1 and n_cells % ncx == 0:
            out.append((ncx, n_cells // ncx))
    return out


def structured_grid(conn, n_nodes):
    """
    The logical grid of a structured mesh (any element type of the library), or None: the element count
    and the node count fix at most two cell counts ncx x ncy; each is tried with the node numbering of the
    rectangle mesher (grid node (i, j) = i (gy + 1) + j, Q8 without the cell centres) and, for Q4 / Q9, of
    the quarter-plate mesher (i + j (gx + 1)), and accepted if the connectivity matches exactly.
    Returns dict(span, epc (elements per cell), ncx, ncy, gx, gy, gnode (grid node -> FE node, -1 for a
    Q8 cell centre), node_ij (FE node -> grid position)).
    """
    n_el, nen = conn.shape
    if nen not in _LAYOUT or n_el == 0:
        return None
    span, epc = _LAYOUT[nen]
    if n_el % epc:
        return None
    n_cells = n_el // epc
    dev = conn.device
    for ncx, ncy in _candidates(n_cells, n_nodes, span, nen == 8):
        gx, gy = span * ncx, span * ncy
        n_grid = (gx + 1) * (gy + 1)
        lex = torch.arange(n_grid, device=dev)
        numberings = [lex.reshape(gx + 1, gy + 1)]
        if nen in (4, 9):
            numberings.append(lex.reshape(gy + 1, gx + 1).t())
        for ids in numberings:
            if nen == 8:                     # drop the cell centres, renumber the other grid nodes in order
                keep = torch.ones(gx + 1, gy + 1, dtype=torch.bool, device=dev)
                keep[1:gx:2, 1:gy:2] = False
                ids = torch.where(keep, torch.cumsum(keep.reshape(-1), 0).reshape(gx + 1, gy + 1) - 1,
                                  torch.full_like(ids, -1))
            if torch.equal(_grid_conn(ids, ncx, ncy, nen), conn):
                gnode = ids.reshape(-1).to(torch.int32).contiguous()
                node_ij = torch.empty(n_nodes, 2, dtype=torch.int32, device=dev)
                ii = torch.arange(gx + 1, device=dev)[:, None].expand(gx + 1, gy + 1).reshape(-1)
                jj = torch.arange(gy + 1, device=dev)[None, :].expand(gx + 1, gy + 1).reshape(-1)
                present = gnode >= 0
                node_ij[gnode[present].long(), 0] = ii[present].to(torch.int32)
                node_ij[gnode[present].long(), 1] = jj[present].to(torch.int32)
                return dict(span=span, epc=epc, ncx=ncx, ncy=ncy, gx=gx, gy=gy, gnode=gnode,
                            node_ij=node_ij.contiguous())
    return None


# ---------------------------------------------------------------------------------------------
# hierarchy
# ---------------------------------------------------------------------------------------------
class _Level:
    def __init__(self, gx, gy, finer=None, device="cuda", n=None):
        self.gx, self.gy = gx, gy
        self.n_nodes = (gx + 1) * (gy + 1)
        self.n = 2 * self.n_nodes if n is None else n       # level 0: the mesh's DOFs
        i32 = dict(dtype=torch.int32, device=device)
        self.keep = []
        self.grid = _lib.MgGrid()
        self.grid.gx, self.grid.gy = gx, gy
        if finer is not None:
            fgx, fgy = finer.gx, finer.gy
            # line I of this level lies on line min(2 I, fgx) of the finer one; finer line i lies in cell
            # min(i // 2, gx - 1) of this level (computed on the device: no host-to-device copies)
            lx = torch.clamp(2 * torch.arange(gx + 1, **i32), max=fgx)
            ly = torch.clamp(2 * torch.arange(gy + 1, **i32), max=fgy)
            cx = torch.clamp(torch.arange(fgx + 1, **i32) // 2, max=gx - 1)
            cy = torch.clamp(torch.arange(fgy + 1, **i32) // 2, max=gy - 1)
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


class Multigrid:
    """
    V-cycle preconditioner r -> z of one structured mesh.  This object owns the hierarchy's device buffers
    and describes them to the C driver (``dfea_mg``): ``setup`` at every linearisation, ``apply`` one cycle,
    ``pcg`` a whole preconditioned CG solve -- each one call into the library (which releases the GIL, so
    concurrent serving threads do not queue behind one another's launches).
    """

    def __init__(self, mesh, params, degree=CHEB_DEGREE, ratio=CHEB_RATIO, lanczos_steps=LANCZOS_STEPS, graphs=True,
                 bounds_every=0, gather=False):
        """``graphs``: graph-driven mode (set-ups replay a captured graph from the second on, the PCG iterates
        in a device-side loop, one graph launch and one status read per solve); False: every launch issued
        from the host.  Both give the same iterates.  ``bounds_every``: 0 estimates the smoother bounds by
        Lanczos at every set-up; k > 0 at the first set-up and every k-th after it, keeping the last estimates
        in between (a set-up then rebuilds the coarse operators only).  ``gather``: the level-0 products in the
        gather form (2 launches each; the mesh's node incidence is built here) instead of one per colour."""
        g = structured_grid(params["conn"].to(mesh.device), mesh.n_nodes)
        if g is None:
            raise ValueError("preconditioner='multigrid' needs a structured mesh (a logical grid of cells)")
        if not 1 <= degree <= _lib.MG_MAX_DEGREE:
            raise ValueError(f"degree must be in [1, {_lib.MG_MAX_DEGREE}]")
        self.mesh, self.g = mesh, g
        self.degree, self.ratio, self.lanczos_steps = degree, ratio, lanczos_steps
        dev = mesh.device
        inv_perm = torch.empty_like(mesh.perm)
        inv_perm[mesh.perm] = torch.arange(mesh.perm.numel(), device=dev)
        # the elements of cell c are c + k n_cells (k < epc: one quadrilateral, or the lower then the upper
        # triangle), numbered like the mesher's
        n_cells = g["ncx"] * g["ncy"]
        elems = torch.arange(n_cells, device=dev)[:, None] + n_cells * torch.arange(g["epc"], device=dev)[None, :]
        self.cell_slot = inv_perm[elems.reshape(-1)].to(torch.int32).contiguous()
        self.levels = [_Level(g["gx"], g["gy"], None, dev, n=mesh.n_dof)]
        while True:
            f = self.levels[-1]
            if len(self.levels) > 1 and (f.n_nodes <= COARSEST_NODES or (f.gx == 1 and f.gy == 1)):
                break
            self.levels.append(_Level(_coarser(f.gx), _coarser(f.gy), f, dev))
        if len(self.levels) > _lib.MG_MAX_LEVELS:
            raise ValueError("multigrid: too many levels")
        last = self.levels[-1]
        if last.n > int(_lib.load().dfea_mg_dense_max()):
            raise ValueError("multigrid: the coarsest level is too large for the dense solve")
        f64 = dict(dtype=torch.float64, device=dev)
        L = len(self.levels)
        self.Ainv = torch.empty(last.n * last.n, **f64)
        self.dense_work = torch.empty_like(self.Ainv)
        self.coef = torch.zeros(L, 2 * _lib.MG_MAX_DEGREE, **f64)
        self.lscal = torch.zeros(L, 4, **f64)
        self.lhist = torch.zeros(L, 2 * lanczos_steps, **f64)
        self.dot_work = torch.zeros(int(_lib.load().dfea_mg_dot_work()), **f64)
        self.pcg_work = torch.empty(4, self.levels[0].n, **f64)
        self.scal = torch.zeros(4, **f64)
        # graph-driven mode: set-ups replay a captured graph, the PCG iterates in a device-side loop
        self.pcg_state = torch.zeros(16, **f64) if graphs else None
        h = self.h = _lib.Mg()
        h.n_levels, h.degree, h.lanczos_steps, h.span, h.ratio = L, degree, lanczos_steps, g["span"], float(ratio)
        h.node_ij, h.gnode, h.cell_slot = g["node_ij"].data_ptr(), g["gnode"].data_ptr(), self.cell_slot.data_ptr()
        for l, lv in enumerate(self.levels):
            dst = h.level[l]
            dst.grid = lv.grid
            dst.n = lv.n
            for name in ("diag", "b", "x", "r", "d", "q"):
                setattr(dst, name, getattr(lv, name).data_ptr())
        for name in ("Ainv", "dense_work", "coef", "lscal", "lhist", "dot_work", "scal"):
            setattr(h, name, getattr(self, name).data_ptr())
        h.pcg = self.pcg_work.data_ptr()
        h.pcg_state = self.pcg_state.data_ptr() if graphs else None
        h.graphs = None
        h.bounds_every, h.setups = int(bounds_every), 0
        self.fe_work = None
        if gather:
            mesh.ensure_node_incidence()
            self.fe_work = torch.empty(int(_lib.load().dfea_gather_work_bytes(mesh.view_ref, _lib.DFEA_F64)),
                                       dtype=torch.uint8, device=dev)
            h.fe_work = self.fe_work.data_ptr()
        self.C, self.code = None, None
        self.id = ops.register_handle(self)
        self.generation = 0          # set-ups so far: a preconditioner closure checks that it is still current

    @property
    def ref(self):
        return ctypes.byref(self.h)

    def setup(self, C, moduli_code, diag):
        """Coarse operators from the fine moduli C (DFEA_F64 / DFEA_F32 / DFEA_F32REF) and the Jacobi diagonal
        (custom op mg_setup)."""
        self.C, self.code = C, moduli_code
        self.generation += 1
        lam = torch.ops.difffea_b200.mg_setup(self.id, C, int(moduli_code), diag).tolist()
        for lv, x in zip(self.levels[:-1], lam):
            lv.lam = x

    def apply(self, r, z):
        """z = M^-1 r (one V-cycle, custom op mg_vcycle); r and z are (2N,) float64 device vectors."""
        z.copy_(torch.ops.difffea_b200.mg_vcycle(self.id, self.C, int(self.code), r.contiguous()))
        return z

    def __call__(self, r):
        return torch.ops.difffea_b200.mg_vcycle(self.id, self.C, int(self.code), r.contiguous())

    def close(self):
        """Release the CUDA graphs the library captured for this hierarchy (graph-driven mode)."""
        h = getattr(self, "h", None)
        if h is not None and h.graphs:
            _lib.load().dfea_mg_release(ctypes.byref(h))

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def pcg(self, b, x, rtol, max_iter):
        """x = PCG(A, b) with the V-cycle, x0 = 0 (custom op mg_pcg); returns (iterations, status name)."""
        it, st = torch.ops.difffea_b200.mg_pcg(self.id, self.C, int(self.code), b, x, float(rtol), int(max_iter)).tolist()
        return it, _lib.PCG_STATUS.get(st, str(st))
