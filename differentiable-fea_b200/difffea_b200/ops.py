"""
PyTorch custom ops over the C ABI (namespace ``difffea_b200``).

Each op is a thin shim: it allocates its outputs through torch's caching allocator and calls one
``extern "C"`` launcher on torch's current stream.  The mesh is referred to by an integer id
(``register_mesh``) because a mesh is a bundle of device arrays, not one tensor.

    torch.ops.difffea_b200.qp_moduli(mesh_id, u, theta, model, scalable, mat_p, fp32, with_diag) -> (C, diag)
    torch.ops.difffea_b200.tangent_apply(mesh_id, C, v) -> y               kernel (b)
    torch.ops.difffea_b200.residual(mesh_id, u, theta, model, scalable, mat_p, f, load_factor) -> (R, |R|^2, energy)
    torch.ops.difffea_b200.element_sensitivity(mesh_id, u, lam, model, scalable, mat_p) -> g      kernel (d)
    torch.ops.difffea_b200.element_fields(mesh_id, u, theta, model, scalable, mat_p) -> (7, n_el)
    torch.ops.difffea_b200.node_fields(mesh_id, elem) -> (6, N)
    torch.ops.difffea_b200.internal_force(mesh_id, u, theta, model, scalable, mat_p) -> R_int (2N,)
    torch.ops.difffea_b200.pcg_solve(pcg_id, x, rtol, max_iter) -> [iterations, status]      kernel (c)
    torch.ops.difffea_b200.mg_setup(mg_id, C, moduli_code, diag) -> lambda_max per smoothed level
    torch.ops.difffea_b200.mg_vcycle(mg_id, C, moduli_code, r) -> z
    torch.ops.difffea_b200.mg_pcg(mg_id, C, moduli_code, b, x, rtol, max_iter) -> [iterations, status]
    torch.ops.difffea_b200.newton_solve(ws_id, theta, n_load_steps, tol, max_newton, max_cutbacks,
                                        pcg_max_iter) -> (u, [converged, load factor, Newton, CG, cut-backs])
and three forms that write into caller buffers, for the solver's preallocated workspace:
    torch.ops.difffea_b200.residual_out(mesh_id, u, theta, model, scalable, mat_p, f, load_factor, R!, scal!, energy)
    torch.ops.difffea_b200.qp_moduli_out(mesh_id, u, theta, model, scalable, mat_p, C!, moduli_code, diag!, blocks!)
    torch.ops.difffea_b200.add_scaled_out(a, alpha, b, out!)                                  out = a + alpha b

The material is (model, scalable, mat_p): the fields of the C ABI's ``dfea_material``
(``material_args`` turns a ``_lib.Material`` into them).  Solver handles -- a device PCG bound to its
buffers (krylov.DevicePCG), a multigrid hierarchy (multigrid.Multigrid), a Newton workspace
(workspace.NewtonWorkspace) -- are referred to by integer ids (``register_handle``) like meshes; the ops that
run them read the buffers the handle is bound to and write the tensors they declare as mutated.
"""
import weakref

import torch

from difffea_b200 import _lib
from difffea_b200.cuda_mesh import ptr, stream_handle

_MESHES = weakref.WeakValueDictionary()


def register_mesh(mesh):
    """Integer handle of a CudaMesh for the custom ops (kept while the mesh is alive)."""
    key = id(mesh)
    _MESHES[key] = mesh
    return key


_HANDLES = weakref.WeakValueDictionary()


def register_handle(obj):
    """Integer id of a solver handle (DevicePCG, Multigrid, NewtonWorkspace) for the custom ops."""
    key = id(obj)
    _HANDLES[key] = obj
    return key


def _handle(handle_id):
    obj = _HANDLES.get(handle_id)
    if obj is None:
        raise RuntimeError(f"unknown or released solver handle {handle_id}")
    return obj


def _mesh(mesh_id):
    mesh = _MESHES.get(mesh_id)
    if mesh is None:
        raise RuntimeError(f"unknown or released mesh id {mesh_id}")
    return mesh


def material_args(mat):
    """(model, scalable, mat_p) of a ``_lib.Material``: the material arguments of the ops."""
    return int(mat.model), int(mat.scalable), [float(x) for x in mat.p]


def _material(model, scalable, mat_p):
    out = _lib.Material()
    out.model, out.scalable = model, scalable
    if len(mat_p) > _lib.MAX_MAT_PARAMS:
        raise ValueError("too many material parameters")
    for k, x in enumerate(mat_p):
        out.p[k] = x
    return out


def _f64(t, mesh, n=None):
    if t.device != mesh.device or t.dtype != torch.float64 or not t.is_contiguous():
        raise ValueError("expected a contiguous float64 tensor on the mesh's device")
    if n is not None and t.numel() != n:
        raise ValueError(f"expected {n} entries, got {t.numel()}")
    return t


@torch.library.custom_op("difffea_b200::qp_moduli", mutates_args=(), device_types="cuda")
def qp_moduli(mesh_id: int, u: torch.Tensor, theta: torch.Tensor, model: int, scalable: int, mat_p: list[float],
              fp32: bool, with_diag: bool) -> tuple[torch.Tensor, torch.Tensor]:
    mesh = _mesh(mesh_id)
    _f64(u, mesh, mesh.n_dof)
    _f64(theta, mesh, mesh.n_el)
    C = torch.empty(mesh.moduli_numel(), dtype=torch.float32 if fp32 else torch.float64, device=mesh.device)
    diag = torch.empty(mesh.n_dof if with_diag else 0, dtype=torch.float64, device=mesh.device)
    _lib.call("dfea_qp_moduli_mat", mesh.view_ref, ptr(u), ptr(theta), _material(model, scalable, mat_p), ptr(C),
              _lib.DFEA_F32 if fp32 else _lib.DFEA_F64, ptr(diag) if with_diag else ptr(None), ptr(None),
              stream_handle())
    return C, diag


@qp_moduli.register_fake
def _(mesh_id, u, theta, model, scalable, mat_p, fp32, with_diag):
    mesh = _mesh(mesh_id)
    C = u.new_empty(mesh.moduli_numel(), dtype=torch.float32 if fp32 else torch.float64)
    return C, u.new_empty(mesh.n_dof if with_diag else 0)


@torch.library.custom_op("difffea_b200::tangent_apply", mutates_args=(), device_types="cuda")
def tangent_apply(mesh_id: int, C: torch.Tensor, v: torch.Tensor) -> torch.Tensor:
    mesh = _mesh(mesh_id)
    fp32 = v.dtype == torch.float32
    if C.dtype == torch.float32:
        mesh.ensure_grad32()
    if v.device != mesh.device or not v.is_contiguous() or v.numel() != mesh.n_dof:
        raise ValueError("v must be a contiguous (2N,) tensor on the mesh's device")
    y = torch.empty_like(v)
    dt = _lib.DFEA_F32 if fp32 else _lib.DFEA_F64
    cdt = _lib.DFEA_F32 if C.dtype == torch.float32 else _lib.DFEA_F64
    _lib.call("dfea_tangent_apply", mesh.view_ref, ptr(C), cdt, ptr(v), ptr(y), dt, stream_handle())
    return y


@tangent_apply.register_fake
def _(mesh_id, C, v):
    return torch.empty_like(v)


@torch.library.custom_op("difffea_b200::residual", mutates_args=(), device_types="cuda")
def residual(mesh_id: int, u: torch.Tensor, theta: torch.Tensor, model: int, scalable: int, mat_p: list[float],
             f: torch.Tensor, load_factor: float) -> tuple[torch.Tensor, torch.Tensor, torch.Tensor]:
    mesh = _mesh(mesh_id)
    _f64(u, mesh, mesh.n_dof)
    _f64(theta, mesh, mesh.n_el)
    _f64(f, mesh, mesh.n_dof)
    R = torch.empty_like(u)
    out = torch.empty(2, dtype=torch.float64, device=mesh.device)
    _lib.call("dfea_residual_mat", mesh.view_ref, ptr(u), ptr(theta), _material(model, scalable, mat_p), ptr(f),
              load_factor, ptr(R), ptr(out), ptr(out[1:]), ptr(mesh.reduce_work()), stream_handle())
    return R, out[0].clone(), out[1].clone()


@residual.register_fake
def _(mesh_id, u, theta, model, scalable, mat_p, f, load_factor):
    return torch.empty_like(u), u.new_empty(()), u.new_empty(())


@torch.library.custom_op("difffea_b200::element_sensitivity", mutates_args=(), device_types="cuda")
def element_sensitivity(mesh_id: int, u: torch.Tensor, lam: torch.Tensor, model: int, scalable: int,
                        mat_p: list[float]) -> torch.Tensor:
    mesh = _mesh(mesh_id)
    _f64(u, mesh, mesh.n_dof)
    _f64(lam, mesh, mesh.n_dof)
    g = torch.empty(mesh.n_el, dtype=torch.float64, device=mesh.device)
    _lib.call("dfea_element_sensitivity_mat", mesh.view_ref, ptr(u), ptr(lam), _material(model, scalable, mat_p),
              ptr(g), stream_handle())
    return g


@element_sensitivity.register_fake
def _(mesh_id, u, lam, model, scalable, mat_p):
    return u.new_empty(_mesh(mesh_id).n_el)


# ---------------------------------------------------------------------------------------------
# post-processing
# ---------------------------------------------------------------------------------------------
@torch.library.custom_op("difffea_b200::element_fields", mutates_args=(), device_types="cuda")
def element_fields(mesh_id: int, u: torch.Tensor, theta: torch.Tensor, model: int, scalable: int,
                   mat_p: list[float]) -> torch.Tensor:
    mesh = _mesh(mesh_id)
    _f64(u, mesh, mesh.n_dof)
    _f64(theta, mesh, mesh.n_el)
    out = torch.empty(7, mesh.n_el, dtype=torch.float64, device=mesh.device)
    _lib.call("dfea_element_fields_mat", mesh.view_ref, ptr(u), ptr(theta), _material(model, scalable, mat_p),
              ptr(out), stream_handle())
    return out


@element_fields.register_fake
def _(mesh_id, u, theta, model, scalable, mat_p):
    return u.new_empty(7, _mesh(mesh_id).n_el)


@torch.library.custom_op("difffea_b200::node_fields", mutates_args=(), device_types="cuda")
def node_fields(mesh_id: int, elem: torch.Tensor) -> torch.Tensor:
    mesh = _mesh(mesh_id)
    if elem.shape != (7, mesh.n_el) or elem.dtype != torch.float64 or not elem.is_contiguous():
        raise ValueError("elem must be the contiguous (7, n_el) float64 output of element_fields")
    mesh.ensure_node_incidence()
    out = torch.empty(6, mesh.n_nodes, dtype=torch.float64, device=mesh.device)
    _lib.call("dfea_node_fields", mesh.view_ref, ptr(elem), ptr(out), stream_handle())
    return out


@node_fields.register_fake
def _(mesh_id, elem):
    return elem.new_empty(6, _mesh(mesh_id).n_nodes)


@torch.library.custom_op("difffea_b200::internal_force", mutates_args=(), device_types="cuda")
def internal_force(mesh_id: int, u: torch.Tensor, theta: torch.Tensor, model: int, scalable: int,
                   mat_p: list[float]) -> torch.Tensor:
    mesh = _mesh(mesh_id)
    _f64(u, mesh, mesh.n_dof)
    _f64(theta, mesh, mesh.n_el)
    R = torch.empty(mesh.n_dof, dtype=torch.float64, device=mesh.device)
    _lib.call("dfea_internal_force_mat", mesh.view_ref, ptr(u), ptr(theta), _material(model, scalable, mat_p),
              ptr(R), stream_handle())
    return R


@internal_force.register_fake
def _(mesh_id, u, theta, model, scalable, mat_p):
    return torch.empty_like(u)


# ---------------------------------------------------------------------------------------------
# solvers
# ---------------------------------------------------------------------------------------------
def _status_tensor(iters, status):
    return torch.tensor([int(iters), int(status)], dtype=torch.int32)


@torch.library.custom_op("difffea_b200::pcg_solve", mutates_args=("x",), device_types="cuda")
def pcg_solve(pcg_id: int, x: torch.Tensor, rtol: float, max_iter: int) -> torch.Tensor:
    """Run a bound device PCG (kernel (c)) on its right-hand side buffer; x must be its solution buffer."""
    import ctypes
    h = _handle(pcg_id)
    if x.data_ptr() != h.x.data_ptr():
        raise ValueError("x must be the solution buffer the PCG handle is bound to")
    iters, status = ctypes.c_int32(0), ctypes.c_int32(0)
    with torch.cuda.device(h.mesh.device):
        _lib.call("dfea_pcg_solve", h._h, float(rtol), int(max_iter), ctypes.byref(iters), ctypes.byref(status),
                  stream_handle())
    return _status_tensor(iters.value, status.value)


@pcg_solve.register_fake
def _(pcg_id, x, rtol, max_iter):
    return torch.empty(2, dtype=torch.int32)


@torch.library.custom_op("difffea_b200::mg_setup", mutates_args=(), device_types="cuda")
def mg_setup(mg_id: int, C: torch.Tensor, moduli_code: int, diag: torch.Tensor) -> torch.Tensor:
    """Set a multigrid hierarchy up at a linearisation (coarse operators, smoother bounds, coarsest inverse)."""
    mg = _handle(mg_id)
    _lib.call("dfea_mg_setup", mg.mesh.view_ref, mg.ref, ptr(C), int(moduli_code), ptr(diag), stream_handle())
    return torch.tensor([float(mg.h.lam[l]) for l in range(len(mg.levels) - 1)], dtype=torch.float64)


@mg_setup.register_fake
def _(mg_id, C, moduli_code, diag):
    return torch.empty(len(_handle(mg_id).levels) - 1, dtype=torch.float64)


@torch.library.custom_op("difffea_b200::mg_vcycle", mutates_args=(), device_types="cuda")
def mg_vcycle(mg_id: int, C: torch.Tensor, moduli_code: int, r: torch.Tensor) -> torch.Tensor:
    mg = _handle(mg_id)
    _f64(r, mg.mesh, mg.mesh.n_dof)
    z = torch.empty_like(r)
    _lib.call("dfea_mg_vcycle", mg.mesh.view_ref, mg.ref, ptr(C), int(moduli_code), ptr(r), ptr(z), stream_handle())
    return z


@mg_vcycle.register_fake
def _(mg_id, C, moduli_code, r):
    return torch.empty_like(r)


@torch.library.custom_op("difffea_b200::mg_pcg", mutates_args=("x",), device_types="cuda")
def mg_pcg(mg_id: int, C: torch.Tensor, moduli_code: int, b: torch.Tensor, x: torch.Tensor, rtol: float,
           max_iter: int) -> torch.Tensor:
    import ctypes
    mg = _handle(mg_id)
    _f64(b, mg.mesh, mg.mesh.n_dof)
    _f64(x, mg.mesh, mg.mesh.n_dof)
    it, st = ctypes.c_int32(0), ctypes.c_int32(0)
    _lib.call("dfea_mg_pcg", mg.mesh.view_ref, mg.ref, ptr(C), int(moduli_code), ptr(b), ptr(x), float(rtol),
              int(max_iter), ctypes.byref(it), ctypes.byref(st), stream_handle())
    return _status_tensor(it.value, st.value)


@mg_pcg.register_fake
def _(mg_id, C, moduli_code, b, x, rtol, max_iter):
    return torch.empty(2, dtype=torch.int32)


@torch.library.custom_op("difffea_b200::newton_solve", mutates_args=(), device_types="cuda")
def newton_solve(ws_id: int, theta: torch.Tensor, n_load_steps: int, tol: float, max_newton: int, max_cutbacks: int,
                 pcg_max_iter: int) -> tuple[torch.Tensor, torch.Tensor]:
    """One complete Newton-Krylov solve by the library's C++ driver on a workspace's buffers."""
    import ctypes
    ws = _handle(ws_id)
    nw, u = ws._native_args(theta)
    info = _lib.NewtonInfo()
    _lib.call("dfea_newton_solve", ctypes.byref(nw), int(n_load_steps), float(tol), int(max_newton), int(max_cutbacks),
              int(pcg_max_iter), ctypes.byref(info), ws._records, ws.MAX_RECORDS, stream_handle())
    stats = torch.tensor([info.converged, info.load_factor, info.total_newton, info.total_cg, info.n_cutbacks,
                          info.n_records], dtype=torch.float64)
    return u, stats


@newton_solve.register_fake
def _(ws_id, theta, n_load_steps, tol, max_newton, max_cutbacks, pcg_max_iter):
    ws = _handle(ws_id)
    return theta.new_empty(ws.mesh.n_dof), torch.empty(6, dtype=torch.float64)


# ---------------------------------------------------------------------------------------------
# the solver workspace's calls, writing into its buffers
# ---------------------------------------------------------------------------------------------
@torch.library.custom_op("difffea_b200::residual_out", mutates_args=("R", "scal"), device_types="cuda")
def residual_out(mesh_id: int, u: torch.Tensor, theta: torch.Tensor, model: int, scalable: int, mat_p: list[float],
                 f: torch.Tensor, load_factor: float, R: torch.Tensor, scal: torch.Tensor, energy: bool) -> None:
    """R = m (R_int(u) - load_factor f); scal[0] = |R|^2 and, with energy, scal[1] = the strain energy."""
    mesh = _mesh(mesh_id)
    _f64(R, mesh, mesh.n_dof)
    if scal.dtype != torch.float64 or scal.numel() < 2 or scal.device != mesh.device:
        raise ValueError("scal must hold at least 2 float64 entries on the mesh's device")
    _lib.call("dfea_residual_mat", mesh.view_ref, ptr(u), ptr(theta), _material(model, scalable, mat_p), ptr(f),
              float(load_factor), ptr(R), ptr(scal), ptr(scal[1:]) if energy else ptr(None),
              ptr(mesh.reduce_work()), stream_handle())


@torch.library.custom_op("difffea_b200::qp_moduli_out", mutates_args=("C", "diag", "blocks"), device_types="cuda")
def qp_moduli_out(mesh_id: int, u: torch.Tensor, theta: torch.Tensor, model: int, scalable: int, mat_p: list[float],
                  C: torch.Tensor, moduli_code: int, diag: torch.Tensor, blocks: torch.Tensor) -> None:
    """Kernel (a) into C (moduli_code layout; empty: the diagonal alone), diag and, when not empty, the inverse
    2x2 node blocks of block-Jacobi."""
    mesh = _mesh(mesh_id)
    _lib.call("dfea_qp_moduli_mat", mesh.view_ref, ptr(u), ptr(theta), _material(model, scalable, mat_p),
              ptr(C) if C.numel() else ptr(None), int(moduli_code), ptr(diag) if diag.numel() else ptr(None),
              ptr(blocks) if blocks.numel() else ptr(None), stream_handle())


@torch.library.custom_op("difffea_b200::add_scaled_out", mutates_args=("out",), device_types="cuda")
def add_scaled_out(a: torch.Tensor, alpha: float, b: torch.Tensor, out: torch.Tensor) -> None:
    """out = a + alpha b (float64): the Newton trial state of the line search."""
    for t in (a, b, out):
        if t.dtype != torch.float64 or not t.is_contiguous() or t.numel() != a.numel() or t.device != a.device:
            raise ValueError("add_scaled_out: contiguous float64 tensors of one size on one device")
    _lib.call("dfea_add_scaled", a.numel(), ptr(a), float(alpha), ptr(b), ptr(out), stream_handle())
