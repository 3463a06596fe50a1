"""
PyTorch custom ops over the C ABI (namespace ``difffea_b200``).

Each op is a thin shim: it allocates its outputs through torch's caching allocator and calls one
``extern "C"`` launcher on torch's current stream.  The mesh is referred to by an integer id
(``register_mesh``) because a mesh is a bundle of device arrays, not one tensor.

    torch.ops.difffea_b200.qp_moduli(mesh_id, u, theta, model, scalable, mat_p, fp32, with_diag) -> (C, diag)
    torch.ops.difffea_b200.tangent_apply(mesh_id, C, v) -> y               kernel (b)
    torch.ops.difffea_b200.residual(mesh_id, u, theta, model, scalable, mat_p, f, load_factor) -> (R, |R|^2, energy)
    torch.ops.difffea_b200.element_sensitivity(mesh_id, u, lam, model, scalable, mat_p) -> g      kernel (d)

The material is (model, scalable, mat_p): the fields of the C ABI's ``dfea_material``
(``material_args`` turns a ``_lib.Material`` into them).
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
