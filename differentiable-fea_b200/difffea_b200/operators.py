"""
Residual, tangent-operator and preconditioner closures on the GPU (the reference's operators.py API).

    global_residual(u, theta, params, load_factor=1.0)          operators.py:159-220
    make_tangent_operator(kind, u, theta, params)               operators.py:415-435, kind "cuda" / "auto"
    make_AT_operator(u, theta, params)                          operators.py:441-471
    compute_jacobi_diagonal / make_jacobi_preconditioner        operators.py:477-570
    make_preconditioner(kind, u, theta, params)                 operators.py:702-710, "jacobi" / "block_jacobi" /
                                                                "multigrid" (structured quad meshes, multigrid.py)
    make_block_jacobi_preconditioner(u, theta, params)          operators.py:586-625
    precompute_geometry(params)                                 operators.py:85-120

Every closure has the reference's semantics -- A(v) = m * J(u)(m * v) + (1 - m) * v, symmetric, the
identity on fixed DOFs -- and runs on the device of ``u`` through the kernels of libdifffea_b200.so.
``"cuda"`` is the stored-moduli variant: kernel (a) evaluates the Gauss-point moduli C once per
linearisation point, kernel (b) applies them.  The reference's own variants (jvp, linearize, qp, qp_ew)
are PyTorch programs of the reference package and are not re-implemented here.
"""
import weakref

import torch

from difffea_b200 import ops
from difffea_b200.cuda_mesh import _require_cuda, cuda_mesh
from difffea_b200.materials import device_material
from difffea_b200.problem import precompute_geometry  # noqa: F401  (re-exported, as in the reference)

TANGENT_OPERATORS = ("auto", "cuda")
REFERENCE_TANGENT_VARIANTS = ("jvp", "linearize", "qp", "qp_ew")
PRECONDITIONERS = ("jacobi", "block_jacobi", "multigrid")


def _prepare(u, theta, params):
    _require_cuda(u, theta)
    mesh = cuda_mesh(params)
    if u.device != mesh.device:
        raise RuntimeError("u and params must be on the same device")
    return mesh, ops.register_mesh(mesh), device_material(params)


def _f64c(t):
    return t.detach().to(torch.float64).contiguous()


# ---------------------------------------------------------------------------------------------
# residual
# ---------------------------------------------------------------------------------------------
def global_residual(u, theta, params, load_factor=1.0):
    """R(u) = m * (R_int(u, theta) - load_factor * f), shape (2N,)."""
    mesh, mid, mat = _prepare(u, theta, params)
    R, _, _ = ops.residual(mid, _f64c(u), _f64c(theta), *ops.material_args(mat), _f64c(params["f"]), float(load_factor))
    return R


def residual_and_norm(u, theta, params, load_factor=1.0):
    """(R, ||R||) with the norm reduced on the device in fixed order (one scalar read-back)."""
    mesh, mid, mat = _prepare(u, theta, params)
    R, n2, _ = ops.residual(mid, _f64c(u), _f64c(theta), *ops.material_args(mat), _f64c(params["f"]),
                            float(load_factor))
    return R, float(n2) ** 0.5


def strain_energy(u, theta, params):
    """Total strain energy sum_e sum_q w detJ psi(F), the ``strain_energy`` of compute_fields."""
    mesh, mid, mat = _prepare(u, theta, params)
    _, _, W = ops.residual(mid, _f64c(u), _f64c(theta), *ops.material_args(mat), _f64c(params["f"]), 0.0)
    return W


# ---------------------------------------------------------------------------------------------
# tangent operator
# ---------------------------------------------------------------------------------------------
class CudaTangentOperator:
    """
    v -> A(v) from moduli stored at the Gauss points (kernel (b)).  Holds the moduli C of its
    linearisation point and the Jacobi diagonal computed in the same pass of kernel (a).
    """

    def __init__(self, mesh, mesh_id, C, diag, precision="fp64"):
        self.mesh, self.mesh_id, self.C, self.diag, self.precision = mesh, mesh_id, C, diag, precision
        self._pcg = None
        self._pcg_diag_src = None
        self.last_status = None

    def __call__(self, v):
        """A(v); FP32 moduli apply to FP32 vectors, or to FP64 vectors with FP64 arithmetic."""
        if v.dtype != self.C.dtype and not (self.C.dtype == torch.float32 and v.dtype == torch.float64):
            raise ValueError(f"this operator applies {self.C.dtype} vectors, got {v.dtype}")
        return ops.tangent_apply(self.mesh_id, self.C, v.contiguous())

    @property
    def dtype(self):
        return self.C.dtype

    def pcg_solve(self, b, diag, rtol, max_iter, preconditioner="jacobi"):
        """
        PCG on the device (kernel (c)) with this operator; returns (x in b's dtype, iterations).  ``diag`` is
        the Jacobi diagonal, or with preconditioner="block_jacobi" the (4N,) inverse node blocks.
        """
        from difffea_b200.krylov import DevicePCG
        vt = b.dtype if self.C.dtype == torch.float32 else torch.float64   # FP32 moduli: FP64 or FP32 vectors
        if preconditioner == "block_jacobi":
            vt = torch.float64
        if (self._pcg is None or self._pcg_diag_src is not diag or self._pcg.vec_dtype != vt
                or self._pcg.preconditioner != preconditioner):
            d = diag.detach().to(vt).contiguous()
            n = self.mesh.n_dof
            bb = torch.empty(n, dtype=vt, device=self.mesh.device)
            xx = torch.empty(n, dtype=vt, device=self.mesh.device)
            if self._pcg is not None:
                self._pcg.close()
            self._pcg = DevicePCG(self.mesh, self.C, d, bb, xx, preconditioner=preconditioner)
            self._pcg_diag_src = diag
        self._pcg.b.copy_(b)
        iters, status = self._pcg.solve(rtol, max_iter)
        self.last_status = status
        return self._pcg.x.to(b.dtype, copy=True), iters


# (weakref(u), u._version, weakref(theta), theta._version, mesh id) -> diag of the last linearisation,
# so that make_preconditioner right after make_tangent_operator at the same point reuses kernel (a)'s pass
_LAST_DIAG = {}


def _diag_key(u, theta, mesh):
    return (id(u), u._version, id(theta), theta._version, id(mesh))


def make_A_operator_cuda(u, theta, params, precision="fp64"):
    """The stored-moduli tangent operator at (u, theta); precision "fp64" or "fp32" (moduli and vectors)."""
    if precision not in ("fp64", "fp32"):
        raise ValueError("precision must be 'fp64' or 'fp32'")
    mesh, mid, mat = _prepare(u, theta, params)
    if precision == "fp32":
        mesh.ensure_grad32()
    C, diag = ops.qp_moduli(mid, _f64c(u), _f64c(theta), *ops.material_args(mat), precision == "fp32", True)
    _LAST_DIAG.clear()
    _LAST_DIAG[_diag_key(u, theta, mesh)] = (weakref.ref(u), weakref.ref(theta), diag)
    return CudaTangentOperator(mesh, mid, C, diag, precision)


def make_tangent_operator(kind, u, theta, params):
    """
    Build the forward tangent operator by name: one of ``TANGENT_OPERATORS``.  "auto" picks "cuda"
    for CUDA tensors (the reference picks qp_ew there and qp on the CPU; its CPU variants stay in the
    reference package).
    """
    if kind == "auto":
        if not u.is_cuda:
            raise RuntimeError("'auto' on a CPU tensor selects the reference's CPU variant 'qp', which lives "
                               "in the reference package; difffea_b200 runs on CUDA devices only")
        kind = "cuda"
    if kind == "cuda":
        return make_A_operator_cuda(u, theta, params)
    if kind in REFERENCE_TANGENT_VARIANTS:
        raise ValueError(f"tangent '{kind}' is one of the reference's PyTorch variants; difffea_b200 provides "
                         f"{TANGENT_OPERATORS}")
    raise ValueError(f"Unknown tangent operator '{kind}'. Choose one of {TANGENT_OPERATORS}.")


def make_AT_operator(u, theta, params):
    """A^T: the hyperelastic tangent is symmetric, so this is the same stored-moduli operator."""
    return make_A_operator_cuda(u, theta, params)


# ---------------------------------------------------------------------------------------------
# Jacobi preconditioner
# ---------------------------------------------------------------------------------------------
class CudaJacobiPreconditioner:
    """r -> r / diag(K) with diag clamped to >= 1e-6 on free DOFs and 1 on fixed DOFs."""

    def __init__(self, mesh, diag):
        self.mesh, self.diag = mesh, diag

    def __call__(self, r):
        return r / self.diag.to(r.dtype)


def compute_jacobi_diagonal(u, theta, params):
    """diag(K) without forming K (kernel (a)'s element diagonals, scattered by colour), shape (2N,)."""
    mesh, mid, mat = _prepare(u, theta, params)
    hit = _LAST_DIAG.get(_diag_key(u, theta, mesh))
    if hit is not None and hit[0]() is u and hit[1]() is theta:
        return hit[2]
    return _diag_only(mesh, u, theta, mat)


def _diag_only(mesh, u, theta, mat):
    from difffea_b200 import _lib
    u64, th64 = _f64c(u), _f64c(theta)
    diag = torch.empty(mesh.n_dof, dtype=torch.float64, device=mesh.device)
    empty = torch.empty(0, dtype=torch.float64, device=mesh.device)
    torch.ops.difffea_b200.qp_moduli_out(ops.register_mesh(mesh), u64, th64, *ops.material_args(mat), empty,
                                         _lib.DFEA_F64, diag, empty)
    return diag


def make_jacobi_preconditioner(u, theta, params):
    mesh = cuda_mesh(params)
    return CudaJacobiPreconditioner(mesh, compute_jacobi_diagonal(u, theta, params))


class CudaBlockJacobiPreconditioner:
    """
    r -> Binv r per node, Binv the inverse of the node's 2x2 tangent block with identity rows/columns on
    fixed DOFs and + 1e-12 I (operators.py:598-625); ``blocks`` = (Binv00, Binv01, Binv11, 0) per node.
    """

    def __init__(self, mesh, blocks):
        self.mesh, self.blocks = mesh, blocks

    def __call__(self, r):
        B = self.blocks.view(-1, 4).to(r.dtype)
        rn = r.view(-1, 2)
        return torch.stack([B[:, 0] * rn[:, 0] + B[:, 1] * rn[:, 1], B[:, 1] * rn[:, 0] + B[:, 2] * rn[:, 1]],
                           dim=1).reshape(-1)


def compute_block_jacobi(u, theta, params):
    """The (4N,) inverse 2x2 node blocks of the tangent at (u, theta) (kernel (a) with the coupling term)."""
    from difffea_b200 import _lib
    mesh, mid, mat = _prepare(u, theta, params)
    u64, th64 = _f64c(u), _f64c(theta)
    diag = torch.empty(mesh.n_dof, dtype=torch.float64, device=mesh.device)
    blocks = torch.empty(2 * mesh.n_dof, dtype=torch.float64, device=mesh.device)
    torch.ops.difffea_b200.qp_moduli_out(mid, u64, th64, *ops.material_args(mat),
                                         torch.empty(0, dtype=torch.float64, device=mesh.device), _lib.DFEA_F64,
                                         diag, blocks)
    return blocks


def make_block_jacobi_preconditioner(u, theta, params):
    mesh = cuda_mesh(params)
    return CudaBlockJacobiPreconditioner(mesh, compute_block_jacobi(u, theta, params))


class CudaMultigridPreconditioner:
    """
    r -> one V-cycle of the geometric multigrid of a structured mesh (multigrid.py), set up at (u, theta).

    The hierarchy's buffers are shared by every preconditioner of the same mesh (one ``Multigrid`` per mesh),
    while each closure keeps the moduli and diagonal of its own linearisation point: when another set-up
    has overwritten the coarse operators since this closure was made, the call sets them up again from its
    own moduli first, so closures made at different states stay independent, as the reference's are.
    """

    def __init__(self, mg, A):
        self.mg, self.A = mg, A
        self.mesh = mg.mesh
        self.generation = mg.generation

    def refresh(self):
        """Set the shared hierarchy up at this closure's linearisation again if another set-up replaced it."""
        if self.mg.generation != self.generation:
            from difffea_b200 import _lib
            self.mg.setup(self.A.C, _lib.DFEA_F64, self.A.diag)
            self.generation = self.mg.generation

    def __call__(self, r):
        self.refresh()
        return self.mg(r.to(torch.float64))


_MG = {}


def multigrid_for(mesh, params):
    """The (cached) Multigrid hierarchy of a mesh."""
    from difffea_b200.multigrid import Multigrid
    key = id(mesh)
    hit = _MG.get(key)
    if hit is None or hit[0]() is not mesh:
        hit = (weakref.ref(mesh), Multigrid(mesh, params))
        _MG.clear()
        _MG[key] = hit
    return hit[1]


def make_multigrid_preconditioner(u, theta, params):
    A = make_A_operator_cuda(u, theta, params)
    mg = multigrid_for(A.mesh, params)
    from difffea_b200 import _lib
    mg.setup(A.C, _lib.DFEA_F64, A.diag)
    return CudaMultigridPreconditioner(mg, A)


def make_preconditioner(kind, u, theta, params):
    """Build a preconditioner by name: one of ``PRECONDITIONERS``."""
    if kind == "jacobi":
        return make_jacobi_preconditioner(u, theta, params)
    if kind == "multigrid":
        return make_multigrid_preconditioner(u, theta, params)
    if kind == "block_jacobi":
        return make_block_jacobi_preconditioner(u, theta, params)
    if kind == "ilu":
        raise ValueError("preconditioner 'ilu' factorises the assembled matrix on the CPU (SciPy); it is not "
                         "built on the device: use 'jacobi' or 'block_jacobi'")
    raise ValueError(f"Unknown preconditioner '{kind}'. Choose one of {PRECONDITIONERS}.")
