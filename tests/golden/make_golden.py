"""
Generate the golden vectors of the reference implementation (run in the build container, where the
reference package is importable; the GPU box only reads the .npz files this writes).

    python tests/golden/make_golden.py [/path/to/reference/src] [--only plate,gradient]

Every fixture is produced by calling the reference's own public functions on small seeded inputs:
problem dictionaries from build_problem (structured rectangle meshes, as in the reference's
tests/helpers.py small_problem), moduli from _qp_setup, products from the qp / qp_ew / jvp tangent
variants, residuals, Jacobi diagonals, strain energies, complete Newton-Krylov solves and adjoint
sensitivities, and the post-processing fields and support reactions of the operator states and of the
solutions.  File names say what each fixture holds.

Two fixtures feed the reference hand-built problem dictionaries, since its build_problem meshes only
rectangles with one clamped side (problem.py:144-146): the quarter plate with a hole (the mapped Q9 mesh
of difffea_b200.mesh, symmetry rollers on x = 0 and y = 0, a dead traction on x = W; the reference's own
element, quadrature, traction, material and geometry functions make the rest of the dictionary) and an
n x n cell unit-square cantilever with a log-normal per-element stiffness scale.
"""
import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
REF_SRC = sys.argv[1] if len(sys.argv) > 1 and not sys.argv[1].startswith("--") else "/root/reference/src"
sys.path.insert(0, REF_SRC)

from difffea.newton_krylov import newton_krylov_solve  # noqa: E402
from difffea.operators import (_qp_setup, compute_jacobi_diagonal, global_residual,  # noqa: E402
                               make_block_jacobi_preconditioner, make_tangent_operator)
from difffea.postprocess import compute_fields, support_reactions  # noqa: E402
from difffea.problem import build_problem, default_spec  # noqa: E402
from difffea.sensitivity import compute_sensitivity  # noqa: E402
from difffea.adjoint import compute_implicit_vjp, solve_adjoint  # noqa: E402
from difffea.boundary_conditions import boundary_edges, edge_traction_load  # noqa: E402
from difffea.elements import edge_shape_fn, element_quadrature, get_element  # noqa: E402
from difffea.materials import material_vector  # noqa: E402
from difffea.newton_krylov import solve_newton_krylov  # noqa: E402
from difffea.operators import precompute_geometry  # noqa: E402
from difffea.problem import lame_parameters  # noqa: E402

sys.path.insert(0, os.path.join(HERE, "..", "..", "differentiable-fea_b200"))
from difffea_b200.mesh import create_quarter_plate_mesh  # noqa: E402  (the mesh only)

torch.set_num_threads(min(8, os.cpu_count() or 1))
DT = torch.float64
KEYS = ("nodes", "conn", "dN_dX", "w_detJ", "f", "m", "fixed", "u_D", "mat_p")


def problem(element_type, h=0.5, load=(60.0, 0.0), E=2600.0, nu=0.3, **over):
    spec = default_spec("rectangle", element_type, h)
    spec.update(mesher="structured", load_value=load, E=E, nu=nu)
    spec.update(over)
    return build_problem(spec)


def arrays(params):
    return {k: params[k].numpy() for k in KEYS}


def fields(u, theta, p):
    """compute_fields (postprocess.py:70-118) as fields_<name> arrays, and support_reactions (121-137)."""
    out = {"fields_" + k: v.numpy() for k, v in compute_fields(u, theta, p).items()}
    out["reactions"] = support_reactions(u, theta, p).numpy()
    return out


def save(name, **arrs):
    path = os.path.join(HERE, name + ".npz")
    np.savez_compressed(path, **{k: np.asarray(v) for k, v in arrs.items()})
    print("wrote", os.path.relpath(path), {k: np.asarray(v).shape for k, v in arrs.items()})


def operator_case(element_type, h, seed, nonuniform_theta):
    p = problem(element_type, h)
    n_el = p["conn"].shape[0]
    g = torch.Generator().manual_seed(seed)
    n = p["f"].shape[0]
    # 0.02 at h = 0.5 (the reference's tests/test_tangent_operators.py state), scaled with h so that no
    # element of the finer meshes is inverted
    u = 0.04 * h * torch.randn(n, dtype=DT, generator=g) * p["m"]
    v = torch.randn(n, dtype=DT, generator=g)
    theta = (0.5 + torch.rand(n_el, dtype=DT, generator=g)) if nonuniform_theta else torch.ones(n_el, dtype=DT)
    C, _ = _qp_setup(u, theta, p)
    out = dict(arrays(p), u=u.numpy(), v=v.numpy(), theta=theta.numpy(), C=C.numpy(),
               Av_qp_ew=make_tangent_operator("qp_ew", u, theta, p)(v).numpy(),
               Av_qp=make_tangent_operator("qp", u, theta, p)(v).numpy(),
               Av_jvp=make_tangent_operator("jvp", u, theta, p)(v).numpy(),
               R=global_residual(u, theta, p).numpy(),
               R_half=global_residual(u, theta, p, load_factor=0.5).numpy(),
               diag=compute_jacobi_diagonal(u, theta, p).numpy(),
               Minv_block_v=make_block_jacobi_preconditioner(u, theta, p)(v).numpy(),
               energy=np.array(float(compute_fields(u, theta, p)["strain_energy"])), **fields(u, theta, p))
    tag = "theta" if nonuniform_theta else "unit"
    save(f"operator_{element_type}_h{h}_{tag}", **out)


def solve_case(element_type, h, load, n_steps, tol_rel, name, preconditioner="jacobi"):
    p = problem(element_type, h, load=load)
    theta = torch.ones(p["conn"].shape[0], dtype=DT)
    tol = tol_rel * float(torch.norm(p["f"]))
    u, info = newton_krylov_solve(p, theta, n_steps, tol, verbose=False, preconditioner=preconditioner, tangent="qp")
    assert info["converged"]
    hist = info["history"]
    save(name, **arrays(p), theta=theta.numpy(), u_star=u.numpy(), tol=np.array(tol),
         n_load_steps=np.array(n_steps), total_newton=np.array(info["total_newton"]),
         total_cg=np.array(info["total_cg"]), residuals=np.array([r["residual"] for r in hist]),
         cg_iters=np.array([r["cg_iters"] for r in hist]), alphas=np.array([r["alpha"] for r in hist]),
         preconditioner=np.array(preconditioner),
         energy=np.array(float(compute_fields(u, theta, p)["strain_energy"])), **fields(u, theta, p))


def sensitivity_case(element_type, h, name):
    p = problem(element_type, h, load=(50.0, 0.0))
    n_el = p["conn"].shape[0]
    theta = 1.0 + 0.2 * torch.sin(torch.arange(n_el, dtype=DT))
    loss_fn = lambda u: torch.dot(p["f"], u)  # noqa: E731  compliance
    u, g = compute_sensitivity(p, theta, loss_fn, n_load_steps=2, tol=1e-12)
    save(name, **arrays(p), theta=theta.numpy(), u_star=u.numpy(), dL_dtheta=g.numpy())


def plate_problem(n, traction=0.1, radius=1.0, half_width=10.0, grading=3.0, E=1.0, nu=0.3):
    """Quarter plate with a hole as a reference params dictionary (mapped n x n Q9 mesh)."""
    nodes, conn = create_quarter_plate_mesh("quad9", n, n, radius, half_width, grading, dtype=DT)
    N = nodes.shape[0]
    el = get_element("quad9")
    GP, GW = element_quadrature("quad9", dtype=DT)
    tol = 1e-9 * half_width
    fixed = torch.stack([nodes[:, 0] <= tol, nodes[:, 1] <= tol], dim=1).reshape(-1)
    load_nodes = nodes[:, 0] >= half_width - tol
    f = edge_traction_load(nodes, boundary_edges(conn, el["edges"]), edge_shape_fn("quad9"), load_nodes,
                           (traction * half_width, 0.0))
    mu0, lmbda0 = lame_parameters(E, nu)
    mat_p, mat_scalable = material_vector("neo_hookean", {"mu": mu0, "lmbda": lmbda0}, dtype=DT)
    params = {"nodes": nodes, "conn": conn, "shape_fn": el["shape_fn"], "GP": GP, "GW": GW,
              "material": "neo_hookean", "mat_p": mat_p, "mat_scalable": mat_scalable, "f": f.reshape(-1),
              "m": torch.where(fixed, 0.0, 1.0).to(DT), "fixed": fixed, "u_D": torch.zeros(2 * N, dtype=DT),
              "element_type": "quad9"}
    return precompute_geometry(params)


def plate_case(n, n_steps, tol_rel, name):
    p = plate_problem(n)
    theta = torch.ones(p["conn"].shape[0], dtype=DT)
    tol = tol_rel * float(torch.norm(p["f"]))
    u, info = newton_krylov_solve(p, theta, n_steps, tol, verbose=False, preconditioner="jacobi", tangent="qp")
    assert info["converged"]
    save(name, **arrays(p), theta=theta.numpy(), u_star=u.numpy(), tol=np.array(tol),
         n_load_steps=np.array(n_steps), total_newton=np.array(info["total_newton"]),
         total_cg=np.array(info["total_cg"]),
         energy=np.array(float(compute_fields(u, theta, p)["strain_energy"])))


def material_arrays(p):
    return dict(arrays(p), material=np.array(p["material"]), mat_scalable=p["mat_scalable"].numpy())


def material_operator_case(material, element_type, h, seed, scalable=None):
    """operator_case's quantities for another material of the library (materials.py:65-186)."""
    p = problem(element_type, h, material=material)
    if scalable is not None:
        p = dict(p, mat_scalable=torch.tensor(scalable))
    n_el, n = p["conn"].shape[0], p["f"].shape[0]
    g = torch.Generator().manual_seed(seed)
    u = 0.04 * h * torch.randn(n, dtype=DT, generator=g) * p["m"]
    v = torch.randn(n, dtype=DT, generator=g)
    theta = 0.5 + torch.rand(n_el, dtype=DT, generator=g)
    C, _ = _qp_setup(u, theta, p)
    tag = "" if scalable is None else "_partial"
    save(f"material_{material}{tag}_{element_type}_h{h}", **material_arrays(p), u=u.numpy(), v=v.numpy(),
         theta=theta.numpy(), C=C.numpy(), Av_qp_ew=make_tangent_operator("qp_ew", u, theta, p)(v).numpy(),
         R=global_residual(u, theta, p).numpy(), R_half=global_residual(u, theta, p, load_factor=0.5).numpy(),
         diag=compute_jacobi_diagonal(u, theta, p).numpy(),
         Minv_block_v=make_block_jacobi_preconditioner(u, theta, p)(v).numpy(),
         energy=np.array(float(compute_fields(u, theta, p)["strain_energy"])), **fields(u, theta, p))


def material_solve_case(material, element_type, h, load, n_steps, tol):
    """The reference's test_materials.py:67-78 problem: a complete solve with the material, tangent qp."""
    p = problem(element_type, h, load=load, material=material)
    theta = torch.ones(p["conn"].shape[0], dtype=DT)
    u, info = newton_krylov_solve(p, theta, n_steps, tol, verbose=False, tangent="qp")
    assert info["converged"]
    save(f"material_solve_{material}_{element_type}_h{h}", **material_arrays(p), theta=theta.numpy(),
         u_star=u.numpy(), tol=np.array(tol), n_load_steps=np.array(n_steps),
         total_newton=np.array(info["total_newton"]), total_cg=np.array(info["total_cg"]),
         energy=np.array(float(compute_fields(u, theta, p)["strain_energy"])), **fields(u, theta, p))


def material_sensitivity_case(material, scalable=None):
    """The reference's test_materials.py:101-114 problem (quad4, h = 1, load (60, 0)) for a material."""
    p = problem("quad4", 1.0, load=(60.0, 0.0), material=material)
    if scalable is not None:
        p = dict(p, mat_scalable=torch.tensor(scalable))
    n_el = p["conn"].shape[0]
    theta = 1.0 + 0.2 * torch.sin(torch.arange(n_el, dtype=DT))
    loss_fn = lambda u: torch.dot(p["f"], u)  # noqa: E731  compliance
    u, g = compute_sensitivity(p, theta, loss_fn, n_load_steps=2, tol=1e-12)
    tag = "" if scalable is None else "_partial"
    save(f"material_sensitivity_{material}{tag}_quad4_h1", **material_arrays(p), theta=theta.numpy(),
         u_star=u.numpy(), dL_dtheta=g.numpy())


OTHER_MATERIALS = ("mooney_rivlin", "saint_venant", "demiray", "fiber_reinforced")


def material_cases():
    for i, mat in enumerate(OTHER_MATERIALS):
        material_operator_case(mat, "quad4", 0.25, seed=10 + i)
        material_operator_case(mat, "quad9", 0.5, seed=20 + i)
        material_operator_case(mat, "tri6", 0.5, seed=30 + i)
        material_solve_case(mat, "quad4", 0.5, (0.0, -15.0), 3, 1e-9)
        material_sensitivity_case(mat)
    # theta scaling only some of the parameters: mu alone (neo-Hookean), mu and k1 (fibre-reinforced)
    material_operator_case("neo_hookean", "quad4", 0.25, seed=40, scalable=[True, False])
    material_sensitivity_case("neo_hookean", scalable=[True, False])
    material_sensitivity_case("fiber_reinforced", scalable=[True, False, True, False, False, False, False])


def gradient_case(n, shear, name, adjoint_max_iter=20000):
    """Unit-square cantilever, n x n Q4, theta = exp(0.3 z) seeded, dead tip shear; compliance gradient."""
    spec = default_spec("rectangle", "quad4", 1.0 / n)
    spec.update(mesher="structured", load_value=(0.0, -shear), E=1.0, nu=0.3)
    spec["geom_params"] = dict(width=1.0, height=1.0)
    p = build_problem(spec)
    assert p["conn"].shape[0] == n * n
    z = torch.randn(n * n, dtype=DT, generator=torch.Generator().manual_seed(0))
    theta = torch.exp(0.3 * z)
    tol = 1e-11 * float(torch.norm(p["f"]))
    u = solve_newton_krylov(p, theta, n_load_steps=1, tol=tol, verbose=False)
    # compute_sensitivity's steps with an adjoint iteration cap that does not bind (its default of 500
    # stops short of rtol 1e-10 at this size)
    lam, k = solve_adjoint(u, theta, p, p["f"], rtol=1e-10, max_iter=adjoint_max_iter)
    assert k < adjoint_max_iter
    g = compute_implicit_vjp(u, theta, p, lam)
    save(name, **arrays(p), theta=theta.numpy(), u_star=u.numpy(), tol=np.array(tol), lam=lam.numpy(),
         adjoint_iters=np.array(k), dL_dtheta=g.numpy(), compliance=np.array(float(torch.dot(p["f"], u))))


def main():
    only = next((a.split("=", 1)[1] if "=" in a else sys.argv[sys.argv.index(a) + 1]
                 for a in sys.argv[1:] if a.startswith("--only")), None)
    if only is not None:
        for what in only.split(","):
            EXTRA[what]()
        return
    for et in ("quad4", "quad8", "quad9", "tri3", "tri6"):
        operator_case(et, 0.5, seed=0, nonuniform_theta=False)
        operator_case(et, 0.25, seed=1, nonuniform_theta=True)
    operator_case("quad4", 0.1, seed=3, nonuniform_theta=True)          # 20 x 10 cells
    # complete solves (the reference's jacobi-PCG path, tangent qp)
    solve_case("quad4", 0.25, (0.0, -40.0), 3, 1e-11, "solve_quad4_h0.25_cantilever")   # dolfinx case
    solve_case("tri6", 0.5, (0.0, -40.0), 3, 1e-11, "solve_tri6_h0.5_cantilever")       # dolfinx case
    solve_case("quad9", 0.5, (0.0, -40.0), 3, 1e-9, "solve_quad9_h0.5_cantilever")
    solve_case("quad4", 0.2, (60.0, 0.0), 2, 1e-10, "solve_quad4_h0.2_tension")
    sensitivity_case("quad4", 1.0, "sensitivity_quad4_h1")
    sensitivity_case("tri3", 1.0, "sensitivity_tri3_h1")
    sensitivity_case("quad4", 0.25, "sensitivity_quad4_h0.25")
    for f in EXTRA.values():
        f()


EXTRA = {
    # the mixed-precision study's geometry at a size the reference solves in under a minute on the CPU
    "plate": lambda: plate_case(24, 5, 1e-11, "plate_quad9_24x24"),
    # the differentiation study's torch.func parity case (128 x 128 cells)
    "gradient": lambda: gradient_case(128, 0.0072, "gradient_quad4_128x128"),
    # nodal block-Jacobi (operators.py:586-625) inside the reference's own Newton-Krylov solve
    "block_jacobi": lambda: (solve_case("quad4", 0.2, (60.0, 0.0), 2, 1e-10, "solve_quad4_h0.2_tension_bj",
                                        preconditioner="block_jacobi"),
                             solve_case("quad9", 0.5, (0.0, -40.0), 3, 1e-9, "solve_quad9_h0.5_cantilever_bj",
                                        preconditioner="block_jacobi")),
    # the other materials of the library: operators, solves and sensitivities
    "materials": material_cases,
    # incomplete-LU preconditioned PCG (operators.py:680-699), the oracle's solver for the large serving requests
    "ilu": lambda: (solve_case("quad4", 0.2, (60.0, 0.0), 2, 1e-10, "solve_quad4_h0.2_tension_ilu",
                               preconditioner="ilu"),
                    solve_case("quad9", 0.5, (0.0, -40.0), 3, 1e-9, "solve_quad9_h0.5_cantilever_ilu",
                               preconditioner="ilu")),
}


if __name__ == "__main__":
    main()
