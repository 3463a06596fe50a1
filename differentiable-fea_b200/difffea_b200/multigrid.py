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

import numpy as np
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
    Connectivity of an ncx x ncy cell grid over the grid node ids (a numpy array), in the element library's
    local order: Q4 / Q9 / Q8 one element per cell, Tri3 / Tri6 the lower-left triangles of all cells, then
    the upper-right ones.
    """
    if nen in (4, 3):
        c = [ids[:ncx, :ncy], ids[1:ncx + 1, :ncy], ids[1:ncx + 1, 1:ncy + 1], ids[:ncx, 1:ncy + 1]]
        q4 = np.stack([t.reshape(-1) for t in c], axis=1)
        return q4 if nen == 4 else np.concatenate([q4[:, [0, 1, 3]], q4[:, [1, 2, 3]]], axis=0)
    offs = [(0, 0), (2, 0), (2, 2), (0, 2), (1, 0), (2, 1), (1, 2), (0, 1), (1, 1)]
    q9 = np.stack([ids[di:di + 2 * ncx:2, dj:dj + 2 * ncy:2].reshape(-1) for di, dj in offs], axis=1)
    if nen == 9:
        return q9
    if nen == 8:
        return q9[:, :8]
    return np.concatenate([q9[:, [0, 1, 3, 4, 8, 7]], q9[:, [1, 2, 3, 5, 6, 8]]], axis=0)


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
    the quarter-plate mesher (i + j (gx + 1)), and accepted if the connectivity matches exactly.  The
    candidate connectivity is built on the host and compared with ``conn`` where it lies (one comparison).
    Returns dict(span, epc (elements per cell), ncx, ncy, gx, gy, gnode (grid node -> FE node, -1 for a
    Q8 cell centre), node_ij (FE node -> grid position)), the tensors on ``conn``'s device.
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
        lex = np.arange((gx + 1) * (gy + 1), dtype=np.int64)
        numberings = [lex.reshape(gx + 1, gy + 1)]
        if nen in (4, 9):
            numberings.append(lex.reshape(gy + 1, gx + 1).T)
        for ids in numberings:
            if nen == 8:                     # drop the cell centres, renumber the other grid nodes in order
                keep = np.ones((gx + 1, gy + 1), dtype=bool)
                keep[1:gx:2, 1:gy:2] = False
                ids = np.where(keep, np.cumsum(keep.reshape(-1)).reshape(gx + 1, gy + 1) - 1, -1)
            expect = _grid_conn(ids, ncx, ncy, nen)
            if expect.shape != tuple(conn.shape) or not torch.equal(torch.from_numpy(expect).to(dev), conn):
                continue
            gnode = ids.reshape(-1).astype(np.int32)
            node_ij = np.empty((n_nodes, 2), dtype=np.int32)
            present = gnode >= 0
            node_ij[gnode[present], 0] = np.repeat(np.arange(gx + 1, dtype=np.int32), gy + 1)[present]
            node_ij[gnode[present], 1] = np.tile(np.arange(gy + 1, dtype=np.int32), gx + 1)[present]
            return dict(span=span, epc=epc, ncx=ncx, ncy=ncy, gx=gx, gy=gy, gnode=torch.from_numpy(gnode).to(dev),
                        node_ij=torch.from_numpy(node_ij).to(dev))
    return None


# ---------------------------------------------------------------------------------------------
# hierarchy
# ---------------------------------------------------------------------------------------------
class _Level:
    """One level's grid (its buffers live in the hierarchy's arenas; ``grid`` holds their addresses)."""

    def __init__(self, gx, gy, n=None):
        self.gx, self.gy = gx, gy
        self.n_nodes = (gx + 1) * (gy + 1)
        self.n = 2 * self.n_nodes if n is None else n       # level 0: the mesh's DOFs
        self.grid = _lib.MgGrid()
        self.grid.gx, self.grid.gy = gx, gy
        self.lam = 1.0

    @property
    def ref(self):
        return ctypes.byref(self.grid)


class _Arena:
    """Offsets of the pieces of one device buffer, each aligned to 256 bytes."""

    def __init__(self, itemsize):
        self.itemsize, self.size, self.at = itemsize, 0, {}

    def add(self, key, count):
        align = 256 // self.itemsize
        self.at[key] = (self.size, count)
        self.size += (count + align - 1) // align * align
        return self.at[key][0]


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
        self.levels = [_Level(g["gx"], g["gy"], n=mesh.n_dof)]
        while True:
            f = self.levels[-1]
            if len(self.levels) > 1 and (f.n_nodes <= COARSEST_NODES or (f.gx == 1 and f.gy == 1)):
                break
            self.levels.append(_Level(_coarser(f.gx), _coarser(f.gy)))
        if len(self.levels) > _lib.MG_MAX_LEVELS:
            raise ValueError("multigrid: too many levels")
        last = self.levels[-1]
        if last.n > int(_lib.load().dfea_mg_dense_max()):
            raise ValueError("multigrid: the coarsest level is too large for the dense solve")
        L = len(self.levels)
        # Integer maps, built on the host and copied in one transfer: the element slot of every cell's elements
        # (cell c holds elements c + k n_cells, k < epc: one quadrilateral, or the lower then the upper
        # triangle, numbered like the mesher's) and per coarse level its line and cell maps -- line I of a
        # level lies on line min(2 I, fgx) of the finer one, finer line i lies in cell min(i // 2, gx - 1).
        n_cells = g["ncx"] * g["ncy"]
        inv_perm = np.empty_like(mesh.perm_host)
        inv_perm[mesh.perm_host] = np.arange(mesh.perm_host.size)
        elems = np.arange(n_cells)[:, None] + n_cells * np.arange(g["epc"])[None, :]
        pieces = {"cell_slot": inv_perm[elems.reshape(-1)]}
        for l in range(1, L):
            f, lv = self.levels[l - 1], self.levels[l]
            pieces[(l, "line_x")] = np.minimum(2 * np.arange(lv.gx + 1), f.gx)
            pieces[(l, "line_y")] = np.minimum(2 * np.arange(lv.gy + 1), f.gy)
            pieces[(l, "cell_x")] = np.minimum(np.arange(f.gx + 1) // 2, lv.gx - 1)
            pieces[(l, "cell_y")] = np.minimum(np.arange(f.gy + 1) // 2, lv.gy - 1)
        ia = _Arena(4)
        for k, v in pieces.items():
            ia.add(k, v.size)
        host = np.zeros(ia.size, dtype=np.int32)
        for k, v in pieces.items():
            o, c = ia.at[k]
            host[o:o + c] = v
        self._ints = torch.from_numpy(host).to(dev)
        # Float64 buffers in one allocation, the zero-initialised ones first: coefficients, Lanczos scalars and
        # history, dot partials, PCG scalars and the graph-driven loop's state; then the coarsest inverse and
        # its work, the PCG vectors and every level's vectors and element matrices.
        fa = _Arena(8)
        fa.add("coef", L * 2 * _lib.MG_MAX_DEGREE)
        fa.add("lscal", L * 4)
        fa.add("lhist", L * 2 * lanczos_steps)
        fa.add("dot_work", int(_lib.load().dfea_mg_dot_work()))
        fa.add("scal", 4)
        if graphs:
            fa.add("pcg_state", 16)
        zero_end = fa.size
        fa.add("Ainv", last.n * last.n)
        fa.add("dense_work", last.n * last.n)
        fa.add("pcg", 4 * self.levels[0].n)
        for l, lv in enumerate(self.levels):
            for name in ("diag", "b", "x", "r", "d", "q"):
                fa.add((l, name), lv.n)
            if l > 0:
                fa.add((l, "K"), 64 * lv.gx * lv.gy)
        self._f64 = torch.empty(fa.size, dtype=torch.float64, device=dev)
        self._f64[:zero_end].zero_()
        ba = _Arena(1)
        for l in range(1, L):
            ba.add(l, self.levels[l].n_nodes)
        self._fix = torch.empty(max(ba.size, 1), dtype=torch.uint8, device=dev)
        self._fa = fa
        ib, fb, bb = self._ints.data_ptr(), self._f64.data_ptr(), self._fix.data_ptr()
        iptr = lambda k: ib + 4 * ia.at[k][0]
        fptr = lambda k: fb + 8 * fa.at[k][0]
        h = self.h = _lib.Mg()
        h.n_levels, h.degree, h.lanczos_steps, h.span, h.ratio = L, degree, lanczos_steps, g["span"], float(ratio)
        h.node_ij, h.gnode, h.cell_slot = g["node_ij"].data_ptr(), g["gnode"].data_ptr(), iptr("cell_slot")
        for l, lv in enumerate(self.levels):
            if l > 0:
                for name in ("line_x", "line_y", "cell_x", "cell_y"):
                    setattr(lv.grid, name, iptr((l, name)))
                lv.grid.K = fptr((l, "K"))
                lv.grid.fix = bb + ba.at[l][0]
            dst = h.level[l]
            dst.grid = lv.grid
            dst.n = lv.n
            for name in ("diag", "b", "x", "r", "d", "q"):
                setattr(dst, name, fptr((l, name)))
        for name in ("Ainv", "dense_work", "coef", "lscal", "lhist", "dot_work", "scal"):
            setattr(h, name, fptr(name))
        h.pcg = fptr("pcg")
        h.pcg_state = fptr("pcg_state") if graphs else None
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

    def buffer(self, name):
        """A view of one of the hierarchy's float64 buffers ("coef", "lscal", "lhist", "Ainv", "pcg", or a level's
        (l, "diag" | "b" | "x" | "r" | "d" | "q" | "K")), for inspection."""
        o, c = self._fa.at[name]
        return self._f64.narrow(0, o, c)

    @property
    def lhist(self):
        """Lanczos coefficients (alpha_k, beta_k) per level, (levels, 2 * lanczos_steps)."""
        return self.buffer("lhist").view(len(self.levels), 2 * self.lanczos_steps)

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
