"""
ctypes binding of libdifffea_b200.so (the C ABI declared in include/difffea_b200.h).

The library is built in-tree by ``differentiable-fea_b200/build.py``.  There is no fallback: if it is
missing or does not load, every compute entry point raises ``RuntimeError`` -- the package never
computes on the CPU or through another implementation behind the caller's back.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libdifffea_b200.so")

DFEA_OK = 0
DFEA_F64 = 0
DFEA_F32 = 1
DFEA_MIXED = 2      # PCG: FP32 moduli/gradients, FP64 Krylov vectors
DFEA_F32REF = 3     # FP32 moduli in the element reference frame (10 per Gauss point), FP64 vectors
MAX_COLOURS = 64

PCG_STATUS = {0: "running", 1: "converged", 2: "max_iter", 3: "negative_curvature", 4: "zero_rhs"}
DFEA_PCG_GATHER = 16  # dfea_pcg_create flag: gather form of the product
DFEA_PCG_BLOCK_JACOBI = 32  # dfea_pcg_create flag: nodal block-Jacobi (diag = inverse 2x2 blocks, 4N)
DFEA_PCG_FUSED = 64  # dfea_pcg_create flag: fused gather form (2 kernels per iteration)


def pcg_max_blocks(n):
    """dfea_pcg_create option: at most n blocks per launch (0: as many as the GPU holds)."""
    if not 0 <= n < 2 ** 23:
        raise ValueError("max_blocks out of range")
    return int(n) << 8

c_i32, c_i64, c_f64, c_vp = ctypes.c_int32, ctypes.c_int64, ctypes.c_double, ctypes.c_void_p


MAX_MAT_PARAMS = 8
DFEA_MAT = {"neo_hookean": 0, "mooney_rivlin": 1, "saint_venant": 2, "demiray": 3, "fiber_reinforced": 4}


class Material(ctypes.Structure):
    """Mirror of ``dfea_material``: model id, theta-scaled parameter bits, nominal parameters."""
    _fields_ = [("model", c_i32), ("scalable", ctypes.c_uint32), ("p", ctypes.c_double * MAX_MAT_PARAMS)]


class MeshView(ctypes.Structure):
    """Mirror of ``dfea_mesh_view``."""
    _fields_ = [
        ("n_el", c_i64), ("stride", c_i64), ("n_nodes", c_i64),
        ("nen", c_i32), ("n_q", c_i32), ("n_colours", c_i32), ("reserved", c_i32),
        ("colour_begin", c_i64 * (MAX_COLOURS + 1)),
        ("conn", c_vp), ("orig", c_vp), ("grad", c_vp), ("wdet", c_vp), ("grad32", c_vp), ("node_fix", c_vp),
        ("node_elem_ptr", c_vp), ("node_elem", c_vp),
        ("jinv", c_vp), ("ref_grad", ctypes.c_double * (9 * 9 * 2)),
    ]


class MgGrid(ctypes.Structure):
    """Mirror of ``dfea_mg_grid``."""
    _fields_ = [("gx", c_i32), ("gy", c_i32), ("line_x", c_vp), ("line_y", c_vp), ("cell_x", c_vp),
                ("cell_y", c_vp), ("K", c_vp), ("fix", c_vp)]


_MGP = ctypes.POINTER(MgGrid)
MG_MAX_LEVELS = 24
MG_MAX_DEGREE = 8


class MgLevel(ctypes.Structure):
    """Mirror of ``dfea_mg_level``."""
    _fields_ = [("grid", MgGrid), ("n", c_i64), ("diag", c_vp), ("b", c_vp), ("x", c_vp), ("r", c_vp), ("d", c_vp),
                ("q", c_vp)]


class Mg(ctypes.Structure):
    """Mirror of ``dfea_mg``."""
    _fields_ = [("n_levels", c_i32), ("degree", c_i32), ("lanczos_steps", c_i32), ("span", c_i32), ("ratio", c_f64),
                ("node_ij", c_vp), ("gnode", c_vp), ("cell_slot", c_vp), ("level", MgLevel * MG_MAX_LEVELS),
                ("Ainv", c_vp), ("dense_work", c_vp), ("coef", c_vp), ("lscal", c_vp), ("lhist", c_vp),
                ("dot_work", c_vp), ("pcg", c_vp), ("scal", c_vp), ("lam", c_f64 * MG_MAX_LEVELS),
                ("pcg_state", c_vp), ("graphs", c_vp), ("bounds_every", c_i32), ("setups", c_i32), ("fe_work", c_vp)]

class Newton(ctypes.Structure):
    """Mirror of ``dfea_newton``: the problem, the buffers and the linear solver of one Newton-Krylov solve."""
    _fields_ = [("mesh", ctypes.POINTER(MeshView)), ("material", Material), ("theta", c_vp), ("f", c_vp),
                ("u_D", c_vp), ("u", c_vp), ("w", c_vp), ("uc", c_vp), ("R", c_vp), ("Rc", c_vp), ("du", c_vp),
                ("b", c_vp), ("diag", c_vp), ("blocks", c_vp), ("moduli", c_vp), ("moduli_dtype", c_i32),
                ("reserved", c_i32), ("reduce_work", c_vp), ("scal", c_vp), ("scal_host", c_vp), ("pcg", c_vp),
                ("mg", ctypes.POINTER(Mg)), ("min_rtol", c_f64)]


class NewtonRecord(ctypes.Structure):
    """Mirror of ``dfea_newton_record``."""
    _fields_ = [("step", c_i32), ("iteration", c_i32), ("cg_iters", c_i32), ("pcg_status", c_i32),
                ("load_factor", c_f64), ("residual", c_f64), ("alpha", c_f64)]


class NewtonInfo(ctypes.Structure):
    """Mirror of ``dfea_newton_info``."""
    _fields_ = [("converged", c_i32), ("total_newton", c_i32), ("total_cg", c_i32), ("n_cutbacks", c_i32),
                ("load_factor", c_f64), ("n_records", c_i32), ("reserved", c_i32)]


class RectSpec(ctypes.Structure):
    """Mirror of ``dfea_rect_spec``: a serving request's structured rectangle for ``dfea_build_rectangle``."""
    _fields_ = [("nen", c_i32), ("n_q", c_i32), ("nx", c_i32), ("ny", c_i32), ("width", c_f64), ("height", c_f64),
                ("load_x", c_f64), ("load_y", c_f64), ("ref_grad", c_f64 * (9 * 9 * 2)), ("gauss_w", c_f64 * 9),
                ("edge_s", c_f64 * 3), ("edge_w", c_f64 * 3)]


_PROTOS = {
    "dfea_last_error": (ctypes.c_char_p, []),
    "dfea_version": (ctypes.c_int, []),
    "dfea_launch_count": (c_i64, []),
    "dfea_set_blocking_sync": (ctypes.c_int, [c_i32, c_i32]),
    "dfea_element_supported": (ctypes.c_int, [c_i32, c_i32]),
    "dfea_struct_size": (c_i64, [ctypes.c_char_p]),
    "dfea_colour_elements": (ctypes.c_int, [c_vp, c_i64, c_i32, c_i64, c_vp, c_vp]),
    "dfea_mesh_pack": (ctypes.c_int, [c_i64, c_i64, c_i32, c_i32, c_i64, c_vp, c_vp, c_vp, c_vp, c_vp,
                                      c_vp, c_vp, c_vp, c_vp, c_vp, c_vp]),
    "dfea_mesh_grad_to_f32": (ctypes.c_int, [ctypes.POINTER(MeshView), c_vp, c_vp]),
    "dfea_mesh_ref_frame": (ctypes.c_int, [ctypes.POINTER(MeshView), c_vp, c_vp, c_vp, c_vp]),
    "dfea_mesh_node_incidence": (ctypes.c_int, [ctypes.POINTER(MeshView), c_vp, c_vp, c_vp, c_vp]),
    "dfea_build_rectangle": (ctypes.c_int, [ctypes.POINTER(RectSpec)] + [c_vp] * 9),
    "dfea_build_rectangle_host": (ctypes.c_int, [ctypes.POINTER(RectSpec)] + [c_vp] * 8),
    "dfea_qp_moduli": (ctypes.c_int, [ctypes.POINTER(MeshView), c_vp, c_vp, c_f64, c_f64, c_vp, c_i32, c_vp, c_vp]),
    "dfea_qp_moduli_block": (ctypes.c_int, [ctypes.POINTER(MeshView), c_vp, c_vp, c_f64, c_f64, c_vp, c_i32, c_vp,
                                            c_vp, c_vp]),
    "dfea_qp_moduli_mat": (ctypes.c_int, [ctypes.POINTER(MeshView), c_vp, c_vp, ctypes.POINTER(Material), c_vp, c_i32,
                                          c_vp, c_vp, c_vp]),
    "dfea_residual_mat": (ctypes.c_int, [ctypes.POINTER(MeshView), c_vp, c_vp, ctypes.POINTER(Material), c_vp, c_f64,
                                         c_vp, c_vp, c_vp, c_vp, c_vp]),
    "dfea_element_sensitivity_mat": (ctypes.c_int, [ctypes.POINTER(MeshView), c_vp, c_vp, ctypes.POINTER(Material),
                                                    c_vp, c_vp]),
    "dfea_element_fields_mat": (ctypes.c_int, [ctypes.POINTER(MeshView), c_vp, c_vp, ctypes.POINTER(Material), c_vp,
                                               c_vp]),
    "dfea_internal_force_mat": (ctypes.c_int, [ctypes.POINTER(MeshView), c_vp, c_vp, ctypes.POINTER(Material), c_vp,
                                               c_vp]),
    "dfea_tangent_apply": (ctypes.c_int, [ctypes.POINTER(MeshView), c_vp, c_i32, c_vp, c_vp, c_i32, c_vp]),
    "dfea_gather_work_bytes": (c_i64, [ctypes.POINTER(MeshView), c_i32]),
    "dfea_tangent_apply_gather": (ctypes.c_int, [ctypes.POINTER(MeshView), c_vp, c_i32, c_vp, c_vp, c_i32, c_vp,
                                                 c_vp]),
    "dfea_reduce_work_bytes": (c_i64, [ctypes.POINTER(MeshView)]),
    "dfea_residual": (ctypes.c_int, [ctypes.POINTER(MeshView), c_vp, c_vp, c_f64, c_f64, c_vp, c_f64, c_vp, c_vp,
                                     c_vp, c_vp, c_vp]),
    "dfea_vec_norm2": (ctypes.c_int, [ctypes.POINTER(MeshView), c_vp, c_vp, c_vp, c_vp]),
    "dfea_element_sensitivity": (ctypes.c_int, [ctypes.POINTER(MeshView), c_vp, c_vp, c_f64, c_f64, c_vp, c_vp]),
    "dfea_element_fields": (ctypes.c_int, [ctypes.POINTER(MeshView), c_vp, c_vp, c_f64, c_f64, c_vp, c_vp]),
    "dfea_node_fields": (ctypes.c_int, [ctypes.POINTER(MeshView), c_vp, c_vp, c_vp]),
    "dfea_internal_force": (ctypes.c_int, [ctypes.POINTER(MeshView), c_vp, c_vp, c_f64, c_f64, c_vp, c_vp]),
    "dfea_mg_galerkin_fe": (ctypes.c_int, [ctypes.POINTER(MeshView), c_vp, c_i32, c_vp, c_vp, c_i32, _MGP, _MGP,
                                           c_vp]),
    "dfea_mg_galerkin": (ctypes.c_int, [_MGP, _MGP, c_vp]),
    "dfea_mg_restrict": (ctypes.c_int, [_MGP, _MGP, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp]),
    "dfea_mg_prolong_add": (ctypes.c_int, [_MGP, _MGP, c_vp, c_vp, c_vp, c_vp, c_vp]),
    "dfea_mg_apply": (ctypes.c_int, [_MGP, c_vp, c_vp, c_vp]),
    "dfea_mg_diag": (ctypes.c_int, [_MGP, c_vp, c_vp]),
    "dfea_mg_cheb_start": (ctypes.c_int, [c_i64, c_vp, c_vp, c_vp, c_vp, c_vp]),
    "dfea_mg_cheb_step": (ctypes.c_int, [c_i64, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_i32, c_vp]),
    "dfea_mg_dot_work": (c_i64, []),
    "dfea_mg_dot": (ctypes.c_int, [c_i64, c_vp, c_vp, c_vp, c_vp, c_vp]),
    "dfea_mg_lanczos_step": (ctypes.c_int, [c_i64, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_i32, c_vp, c_vp]),
    "dfea_mg_dense_max": (c_i64, []),
    "dfea_mg_lanczos_bound": (ctypes.c_double, [c_vp, c_i32]),
    "dfea_mg_setup": (ctypes.c_int, [ctypes.POINTER(MeshView), ctypes.POINTER(Mg), c_vp, c_i32, c_vp, c_vp]),
    "dfea_mg_vcycle": (ctypes.c_int, [ctypes.POINTER(MeshView), ctypes.POINTER(Mg), c_vp, c_i32, c_vp, c_vp, c_vp]),
    "dfea_mg_release": (ctypes.c_int, [ctypes.POINTER(Mg)]),
    "dfea_mg_pcg": (ctypes.c_int, [ctypes.POINTER(MeshView), ctypes.POINTER(Mg), c_vp, c_i32, c_vp, c_vp, c_f64, c_i32,
                                   ctypes.POINTER(c_i32), ctypes.POINTER(c_i32), c_vp]),
    "dfea_mg_dense_inverse": (ctypes.c_int, [_MGP, c_vp, c_vp, c_vp]),
    "dfea_mg_dense_solve": (ctypes.c_int, [c_i32, c_vp, c_vp, c_vp, c_vp]),
    "dfea_batch_create": (ctypes.c_int, [c_i32, c_i32, c_vp]),
    "dfea_batch_destroy": (ctypes.c_int, [c_vp]),
    "dfea_batch_start": (ctypes.c_int, [c_vp, c_vp, c_f64, c_i32, c_vp]),
    "dfea_batch_set": (ctypes.c_int, [c_vp, c_vp, c_i32, c_vp]),
    "dfea_batch_iterate": (ctypes.c_int, [c_vp, c_i32, c_vp, c_vp, c_vp]),
    "dfea_pcg_work_bytes": (c_i64, [ctypes.POINTER(MeshView), c_i32]),
    "dfea_pcg_create": (ctypes.c_int, [ctypes.POINTER(MeshView), c_vp, c_vp, c_vp, c_vp, c_i32, c_vp, c_i32,
                                       ctypes.POINTER(c_vp)]),
    "dfea_pcg_solve": (ctypes.c_int, [c_vp, c_f64, c_i32, ctypes.POINTER(c_i32), ctypes.POINTER(c_i32), c_vp]),
    "dfea_pcg_destroy": (ctypes.c_int, [c_vp]),
    "dfea_pcg_solve_noalloc": (ctypes.c_int, [ctypes.POINTER(MeshView), c_vp, c_vp, c_vp, c_vp, c_i32, c_f64, c_i32,
                                              ctypes.POINTER(c_i32), ctypes.POINTER(c_i32), c_vp]),
    "dfea_newton_solve": (ctypes.c_int, [ctypes.POINTER(Newton), c_i32, c_f64, c_i32, c_i32, c_i32,
                                         ctypes.POINTER(NewtonInfo), ctypes.POINTER(NewtonRecord), c_i32, c_vp]),
    "dfea_axpy": (ctypes.c_int, [c_i64, c_f64, c_vp, c_vp, c_vp]),
    "dfea_add_scaled": (ctypes.c_int, [c_i64, c_vp, c_f64, c_vp, c_vp, c_vp]),
    "dfea_f64_to_f32": (ctypes.c_int, [c_i64, c_vp, c_vp, c_vp]),
    "dfea_f32_to_f64": (ctypes.c_int, [c_i64, c_vp, c_vp, c_vp]),
}

_lib = None
_load_error = None


def exported_symbols():
    """Names of the C entry points this binding expects (the declarations of include/difffea_b200.h)."""
    return sorted(_PROTOS)


def load():
    """Load the library once; raise RuntimeError with the reason if it is not there."""
    global _lib, _load_error
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        _load_error = (f"{LIB_PATH} is missing: build it with `python differentiable-fea_b200/build.py` "
                       "(the CUDA kernels have no fallback)")
        raise RuntimeError(_load_error)
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in _PROTOS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def last_error():
    return load().dfea_last_error().decode(errors="replace")


def check(rc, what):
    """Raise RuntimeError for a non-zero return code of a C entry point."""
    if rc != DFEA_OK:
        raise RuntimeError(f"{what} failed (code {rc}): {last_error()}")


def call(name, *args):
    """Call a C entry point by name and check its return code."""
    rc = getattr(load(), name)(*args)
    check(rc, name)
    return rc
