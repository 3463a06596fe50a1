"""
Post-processing of a converged displacement on the GPU (the reference's postprocess.py API).

    compute_fields(u, theta, params) -> dict         postprocess.py:70-118
    support_reactions(u, theta, params) -> (2,)      postprocess.py:121-137

Per element, one kernel evaluates the Gauss-point state [J, sigma_xx, sigma_yy, sigma_xy, sigma_zz, psi] of
the problem's material (sigma = P3 F3^T / J with F33 = 1, postprocess.py:24-47), averages it
with the physical weights w detJ and writes the element area and von Mises of the averaged components
(postprocess.py:50-67, 96-98).  A second kernel averages the element fields over each node's incident
elements through the node -> element incidence (postprocess.py:109-117); it sums in incidence order
instead of conn order, so nodal values differ from a sequential scatter-add by rounding only.  The
support reactions are the internal force with no mask (every DOF) summed over the fixed DOFs.
"""
import torch

from difffea_b200 import ops
from difffea_b200.operators import _f64c, _prepare

ELEMENT_FIELDS = ("J", "sxx", "syy", "sxy", "mises", "energy_density")


def element_fields(u, theta, params):
    """(7, n_el) per original element: area, then the weighted means J, sxx, syy, sxy, mises, psi."""
    mesh, mid, mat = _prepare(u, theta, params)
    return torch.ops.difffea_b200.element_fields(mid, _f64c(u), _f64c(theta), *ops.material_args(mat))


def compute_fields(u, theta, params) -> dict:
    """
    All post-processing fields of a converged solution, keys as the reference's:
        per element (n_el,):  J, sxx, syy, sxy, mises, energy_density
        per node (N,):        ux, uy, u_mag (and ux_n, uy_n, u_mag_n), and J_n ... energy_density_n
        scalars (0-d):        strain_energy, min_J
    """
    mesh, mid, _ = _prepare(u, theta, params)
    el = element_fields(u, theta, params)
    nodal = torch.ops.difffea_b200.node_fields(mid, el)
    un = _f64c(u).view(mesh.n_nodes, 2)
    out = {name: el[k + 1] for k, name in enumerate(ELEMENT_FIELDS)}
    out.update(ux=un[:, 0], uy=un[:, 1], u_mag=torch.linalg.norm(un, dim=1),
               strain_energy=torch.sum(el[6] * el[0]), min_J=el[1].min())
    for name in ("ux", "uy", "u_mag"):
        out[name + "_n"] = out[name]
    for k, name in enumerate(ELEMENT_FIELDS):
        out[name + "_n"] = nodal[k]
    return out


def internal_force(u, theta, params):
    """R_int(u) at every DOF, the constrained ones included (no mask, no external load)."""
    mesh, mid, mat = _prepare(u, theta, params)
    return torch.ops.difffea_b200.internal_force(mid, _f64c(u), _f64c(theta), *ops.material_args(mat))


def support_reactions(u, theta, params) -> torch.Tensor:
    """Total reaction (Rx, Ry) at the constrained DOFs; sum(reactions) + sum(applied loads) = 0 at equilibrium."""
    R = internal_force(u, theta, params).view(-1, 2)
    fixed = params["fixed"].to(R.device).reshape(-1, 2).bool()
    return torch.sum(torch.where(fixed, R, torch.zeros_like(R)), dim=0)
