"""
Problem set-up: spec dictionary -> ``params`` dictionary (host set-up, then one copy to the device).

``build_problem(spec)`` returns the keys of the reference's problem dictionary (problem.py:115-194,
operators.py:19-34): nodes, conn, shape_fn, GP, GW, material, mat_p, mat_scalable, f, m, fixed, u_D,
element_type, and the cached geometry dN_dX, w_detJ.  A dictionary built by the reference itself is
accepted by every entry point of this package just the same.

Meshing: structured rectangles (the reference's "structured" mesher).  Gmsh geometries are not
built; the mapped quarter plate with a hole has its own builder (``build_quarter_plate_problem``).
"""
import torch

from difffea_b200.boundary_conditions import (boundary_edges, bounding_box, dofs_from_node_mask, edge_traction_load,
                                              select_boundary_nodes)
from difffea_b200.elements import element_quadrature, get_element, make_shape_fn, quadrature_gradients
from difffea_b200.materials import lame_parameters, material_vector
from difffea_b200.mesh import create_quarter_plate_mesh, create_rectangle_mesh

GEOMETRIES = {"rectangle": dict(params=dict(width=2.0, height=1.0))}

GEOMETRY_PRESETS = {
    "rectangle": dict(fixed_side="left", fixed_dofs="xy", load_side="right", load_mode="force",
                      load_value=(0.0, -40.0)),
}


def default_spec(geometry="rectangle", element_type="quad4", h=0.2):
    """A ready-to-run specification (rectangle cantilever, E = 2600, nu = 0.3, structured mesh)."""
    if geometry not in GEOMETRIES:
        raise ValueError(f"geometry '{geometry}' needs Gmsh, which this package does not drive; "
                         f"use one of {list(GEOMETRIES)}")
    return dict(geometry=geometry, geom_params=dict(GEOMETRIES[geometry]["params"]), element_type=element_type,
                h=h, mesher="structured", E=2600.0, nu=0.3, dtype=torch.float64, **GEOMETRY_PRESETS[geometry])


def to_device(params, device):
    """New dictionary with every tensor moved to ``device``."""
    return {k: (v.to(device) if torch.is_tensor(v) else v) for k, v in params.items()}


def precompute_geometry(params):
    """
    dN_dX (n_el, n_q, nen, 2) = J^-T grad_xi N and w_detJ (n_el, n_q) = w det J, with J = dX/dxi the mesh
    Jacobian at every Gauss point (operators.py:85-120), in closed form.  Returns a NEW dictionary.
    """
    nodes, conn, GP, GW = params["nodes"], params["conn"], params["GP"], params["GW"]
    name = params.get("element_type") or getattr(params.get("shape_fn"), "element_type", None)
    if name is None:
        raise ValueError("precompute_geometry needs params['element_type']")
    dNr = quadrature_gradients(name, GP).to(nodes.dtype)                        # (n_q, nen, 2)
    Xe = nodes[conn]                                                            # (n_el, nen, 2)
    J = torch.einsum("eai,qaj->eqij", Xe, dNr)                                  # dX_i / dxi_j
    det = J[..., 0, 0] * J[..., 1, 1] - J[..., 0, 1] * J[..., 1, 0]
    inv = torch.stack([torch.stack([J[..., 1, 1], -J[..., 0, 1]], -1),
                       torch.stack([-J[..., 1, 0], J[..., 0, 0]], -1)], -2) / det[..., None, None]
    dN_dX = torch.einsum("qaj,eqji->eqai", dNr, inv)
    return {**params, "dN_dX": dN_dX.contiguous(), "w_detJ": (GW[None, :] * det).contiguous()}


def _assemble(nodes, conn, element_type, spec, dtype):
    """Boundary conditions, loads and material on the device of ``nodes`` (CPU or GPU)."""
    el = get_element(element_type)
    dev = nodes.device
    GP, GW = element_quadrature(element_type, dtype=dtype, device=dev)
    N = nodes.shape[0]
    box = bounding_box(nodes)
    fixed_nodes = select_boundary_nodes(nodes, spec["fixed_side"], box=box)
    comps = {"xy": (0, 1), "x": (0,), "y": (1,)}[spec.get("fixed_dofs", "xy")]
    fixed = dofs_from_node_mask(fixed_nodes, comps)
    u_D = torch.zeros(2 * N, dtype=dtype, device=dev)
    load_nodes = select_boundary_nodes(nodes, spec["load_side"], box=box)
    value = spec.get("load_value", (0.0, 0.0))
    f = torch.zeros(N, 2, dtype=dtype, device=dev)
    if spec.get("load_mode", "force") == "displacement":
        for c, val in enumerate(value):
            if val is None:
                continue
            mask = dofs_from_node_mask(load_nodes, (c,))
            fixed = fixed | mask
            u_D = torch.where(mask, torch.as_tensor(float(val), dtype=dtype, device=dev), u_D)
    else:
        edges = boundary_edges(conn, el["edges"], node_mask=load_nodes, n_nodes=N)
        f = edge_traction_load(nodes, edges, el["order"], load_nodes, (float(value[0]), float(value[1])))
    m = torch.where(fixed, 0.0, 1.0).to(dtype)
    material = spec.get("material", "neo_hookean")
    values = spec.get("material_params")
    if values is None and material == "neo_hookean" and "E" in spec:
        mu0, lmbda0 = lame_parameters(spec["E"], spec["nu"])
        values = {"mu": mu0, "lmbda": lmbda0}
    mat_p, mat_scalable = material_vector(material, values, dtype=dtype)
    return {"nodes": nodes, "conn": conn, "shape_fn": make_shape_fn(element_type), "GP": GP, "GW": GW,
            "material": material, "mat_p": mat_p.to(dev), "mat_scalable": mat_scalable.to(dev),
            "f": f.reshape(-1), "m": m, "fixed": fixed, "u_D": u_D, "element_type": element_type}


def build_problem(spec):
    """spec -> params (see the module docstring); ``spec["device"]`` moves the result to a GPU."""
    dtype = spec.get("dtype", torch.float64)
    if spec.get("mesher", "structured") != "structured":
        raise ValueError("only the structured mesher is available (Gmsh geometries are not built)")
    if spec["geometry"] != "rectangle":
        raise ValueError("The structured mesher only supports the 'rectangle' geometry.")
    gp = spec["geom_params"]
    nx = max(1, round(gp["width"] / spec["h"]))
    ny = max(1, round(gp["height"] / spec["h"]))
    nodes, conn = create_rectangle_mesh(spec["element_type"], gp["width"], gp["height"], nx, ny, dtype=dtype)
    params = precompute_geometry(_assemble(nodes, conn, spec["element_type"], spec, dtype))
    device = spec.get("device", "cpu")
    return params if str(device) == "cpu" else to_device(params, device)


def build_rectangle_problem(element_type, nx, ny, width, height, E=1.0, nu=0.3, load=(0.0, 0.0),
                            fixed_side="left", load_side="right", fixed_dofs="xy", load_mode="force",
                            device="cpu", dtype=torch.float64, build_on_device=False, material="neo_hookean",
                            material_params=None):
    """
    Rectangle with an exact nx x ny cell count (the spec interface derives counts from h).
    ``build_on_device`` constructs mesh, loads and geometry directly on ``device`` (torch ops there)
    instead of on the host followed by one copy.  ``material`` / ``material_params`` as in the spec
    (neo-Hookean from E and nu when no parameters are given).
    """
    where = device if build_on_device else "cpu"
    nodes, conn = create_rectangle_mesh(element_type, width, height, nx, ny, dtype=dtype, device=where)
    spec = dict(fixed_side=fixed_side, fixed_dofs=fixed_dofs, load_side=load_side, load_mode=load_mode,
                load_value=load, E=E, nu=nu, material=material, material_params=material_params)
    params = precompute_geometry(_assemble(nodes, conn, element_type, spec, dtype))
    return params if str(params["nodes"].device) == str(torch.device(device)) else to_device(params, device)


def build_quarter_plate_problem(element_type="quad9", n_theta=256, n_radial=256, radius=1.0, half_width=10.0,
                                traction=0.1, E=1.0, nu=0.3, grading=3.0, device="cpu", dtype=torch.float64):
    """
    Quarter of a square plate with a central hole under uniaxial tension: symmetry rollers on x = 0
    (u_x = 0) and y = 0 (u_y = 0), a uniform dead traction ``traction`` (force per unit reference length)
    in +x on the edge x = W.
    """
    nodes, conn = create_quarter_plate_mesh(element_type, n_theta, n_radial, radius, half_width, grading,
                                            dtype=dtype)
    N = nodes.shape[0]
    el = get_element(element_type)
    GP, GW = element_quadrature(element_type, dtype=dtype)
    tol = 1e-9 * half_width
    fix_x = nodes[:, 0] <= tol
    fix_y = nodes[:, 1] <= tol
    fixed = torch.stack([fix_x, fix_y], dim=1).reshape(-1)
    load_nodes = nodes[:, 0] >= half_width - tol
    edges = boundary_edges(conn, el["edges"])
    f = edge_traction_load(nodes, edges, el["order"], load_nodes, (traction * half_width, 0.0))
    mu0, lmbda0 = lame_parameters(E, nu)
    mat_p, mat_scalable = material_vector("neo_hookean", {"mu": mu0, "lmbda": lmbda0}, dtype=dtype)
    params = {"nodes": nodes, "conn": conn, "shape_fn": make_shape_fn(element_type), "GP": GP, "GW": GW,
              "material": "neo_hookean", "mat_p": mat_p, "mat_scalable": mat_scalable, "f": f.reshape(-1),
              "m": torch.where(fixed, 0.0, 1.0).to(dtype), "fixed": fixed, "u_D": torch.zeros(2 * N, dtype=dtype),
              "element_type": element_type}
    params = precompute_geometry(params)
    return params if str(device) == "cpu" else to_device(params, device)
