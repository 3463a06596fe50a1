"""
CPU restatement of the reference's Newton-Krylov path (test infrastructure; see oracle/__init__.py).

Inputs are "problem" dictionaries with the reference's keys (operators.py:19-34): nodes (N,2),
conn (n_el,nen) int64, dN_dX (n_el,n_q,nen,2), w_detJ (n_el,n_q), f, m, u_D (2N,) float64,
fixed (2N,) bool, material (name), mat_p (n_p,), mat_scalable (n_p,) bool.  Everything runs in float64 on the CPU with PyTorch's
CPU kernels and torch.func autodiff, i.e. the same arithmetic the reference performs -- which is also
why this module doubles as the reference CPU baseline for timing.
"""
import torch
from torch.func import grad, hessian, jvp, vjp, vmap

F64 = torch.float64


def as_problem(p):
    """CPU float64 copy of the keys the path reads (accepts reference- or package-built dictionaries)."""
    out = {}
    for k in ("nodes", "dN_dX", "w_detJ", "f", "m", "u_D", "mat_p"):
        out[k] = torch.as_tensor(p[k]).detach().to("cpu", F64).contiguous()
    out["conn"] = torch.as_tensor(p["conn"]).detach().to("cpu", torch.int64).contiguous()
    out["fixed"] = torch.as_tensor(p["fixed"]).detach().to("cpu", torch.bool)
    out["material"] = p.get("material", "neo_hookean")
    sc = p.get("mat_scalable")
    out["mat_scalable"] = (torch.ones(out["mat_p"].numel(), dtype=torch.bool) if sc is None
                           else torch.as_tensor(sc).detach().to("cpu", torch.bool))
    return out


# ---------------------------------------------------------------------------------------------
# material: plane-strain neo-Hookean energy (materials.py:181-217, 343-349)
# ---------------------------------------------------------------------------------------------
def psi(F, p):
    """psi(F2, [mu, lambda]) of the embedding F3 = [[F, 0], [0, 1]]: mu/2 (I1 - 3 - 2 lnJ) + lambda/2 lnJ^2."""
    I1 = (F * F).sum() + 1.0                         # tr(F3^T F3), materials.py:215
    J = F[0, 0] * F[1, 1] - F[0, 1] * F[1, 0]        # det F3 = det F2 * 1, materials.py:195-198
    lnJ = torch.log(J)
    return 0.5 * p[0] * (I1 - 3.0 - 2.0 * lnJ) + 0.5 * p[1] * lnJ ** 2


def element_parameters(theta, P):
    """p_e = p0 * theta_e on the scalable parameters, p0 on the others (materials.py:239-246)."""
    factor = torch.where(P["mat_scalable"][None, :], theta[:, None], torch.ones_like(theta)[:, None])
    return P["mat_p"][None, :] * factor


# the other energies of the library (materials.py:65-161), as functions of the 3x3 embedding
def _det3(F3):
    return (F3[0, 0] * F3[1, 1] - F3[0, 1] * F3[1, 0]) * F3[2, 2]       # materials.py:51-54


def _psi3_neo_hookean(F3, p):
    lnJ = torch.log(_det3(F3))
    return 0.5 * p[0] * ((F3 * F3).sum() - 3.0 - 2.0 * lnJ) + 0.5 * p[1] * lnJ ** 2


def _psi3_mooney_rivlin(F3, p):
    C = F3.T @ F3
    I1 = torch.trace(C)
    I2 = 0.5 * (I1 ** 2 - torch.trace(C @ C))
    J = _det3(F3)
    return p[0] * (J ** (-2.0 / 3.0) * I1 - 3.0) + p[1] * (J ** (-4.0 / 3.0) * I2 - 3.0) + 0.5 * p[2] * torch.log(J) ** 2


def _psi3_saint_venant(F3, p):
    E = 0.5 * (F3.T @ F3 - torch.eye(3, dtype=F3.dtype))
    return 0.5 * p[1] * torch.trace(E) ** 2 + p[0] * (E * E).sum()


def _psi3_demiray(F3, p):
    lnJ = torch.log(_det3(F3))
    return p[0] / (2.0 * p[1]) * (torch.exp(p[1] * ((F3 * F3).sum() - 3.0)) - 1.0) - p[0] * lnJ + 0.5 * p[2] * lnJ ** 2


def _psi3_fiber_reinforced(F3, p):
    C = F3.T @ F3
    I1 = torch.trace(C)
    beta = torch.deg2rad(p[4])
    zero = torch.zeros_like(beta)
    total = _psi3_neo_hookean(F3, p[:2])
    for k, sign in enumerate((1.0, -1.0)):
        a = torch.stack([torch.cos(beta), sign * torch.sin(beta), zero])
        E = p[5] * I1 + (1.0 - 3.0 * p[5]) * (a @ C @ a) - 1.0
        fib = p[2] / (2.0 * p[3]) * (torch.exp(p[3] * torch.relu(E) ** 2) - 1.0)
        total = total + (fib if k == 0 else p[6] * fib)
    return total


PSI3 = {"neo_hookean": _psi3_neo_hookean, "mooney_rivlin": _psi3_mooney_rivlin, "saint_venant": _psi3_saint_venant,
        "demiray": _psi3_demiray, "fiber_reinforced": _psi3_fiber_reinforced}


def embed(F):
    """F3 = [[F, 0], [0, 1]] built with stack, so that every autodiff transform sees through it."""
    z, o = torch.zeros_like(F[0, 0]), torch.ones_like(F[0, 0])
    return torch.stack([torch.stack([F[0, 0], F[0, 1], z]), torch.stack([F[1, 0], F[1, 1], z]),
                        torch.stack([z, z, o])])


def energy(P):
    """psi(F2, p) of the problem's material: the closed neo-Hookean form above, else psi3 of the embedding."""
    name = P.get("material", "neo_hookean")
    if name == "neo_hookean":
        return psi
    psi3_fn = PSI3[name]
    return lambda F, p: psi3_fn(embed(F), p)


def gather_nodes(u, conn):
    """(2N,) DOF vector -> (n_el, nen, 2) element values, dof = 2 node + comp (operators.py:186-187)."""
    return u.reshape(-1, 2)[conn]


def scatter_nodes(fe, conn, n_nodes):
    """index_add_ of (n_el, nen, 2) element vectors into a (2N,) vector (operators.py:210-214)."""
    out = torch.zeros(n_nodes, 2, dtype=fe.dtype)
    out.index_add_(0, conn.reshape(-1), fe.reshape(-1, 2))
    return out.reshape(-1)


def deformation_gradient(ue, dN):
    """F = I + sum_a u_a (x) dN_a at every Gauss point (operators.py:334-336)."""
    return torch.eye(2, dtype=F64) + torch.einsum("eai,eqaj->eqij", ue, dN)


# ---------------------------------------------------------------------------------------------
# residual (operators.py:131-220) and strain energy (postprocess.py:70-118, line 102)
# ---------------------------------------------------------------------------------------------
def element_forces(u, theta, P):
    """f_e[a, i] = sum_q w detJ P_ij(F_q) dN_aj, with P = d psi / dF by autodiff (operators.py:151-156)."""
    ue = gather_nodes(u, P["conn"])
    F = deformation_gradient(ue, P["dN_dX"])
    pe = element_parameters(theta, P)
    stress = vmap(vmap(grad(energy(P)), in_dims=(0, None)), in_dims=(0, 0))(F, pe)
    return torch.einsum("eq,eqij,eqaj->eai", P["w_detJ"], stress, P["dN_dX"])


def residual(u, theta, P, load_factor=1.0):
    """R = m * (scatter(f_e) - load_factor f)   (global_residual, operators.py:159-220)."""
    R = scatter_nodes(element_forces(u, theta, P), P["conn"], P["nodes"].shape[0]) - load_factor * P["f"]
    return P["m"] * R


def strain_energy(u, theta, P):
    """sum_e sum_q w detJ psi(F_q) (compute_fields' "strain_energy")."""
    F = deformation_gradient(gather_nodes(u, P["conn"]), P["dN_dX"])
    pe = element_parameters(theta, P)
    dens = vmap(vmap(energy(P), in_dims=(0, None)), in_dims=(0, 0))(F, pe)
    return (dens * P["w_detJ"]).sum()


# ---------------------------------------------------------------------------------------------
# stored-moduli tangent (operators.py:316-412)
# ---------------------------------------------------------------------------------------------
def moduli(u, theta, P):
    """C[e, q] = w detJ * hessian(psi)(F) flattened (ij),(kl) -> 4x4 (_qp_setup, operators.py:316-342)."""
    F = deformation_gradient(gather_nodes(u, P["conn"]), P["dN_dX"])
    pe = element_parameters(theta, P)
    H = vmap(vmap(hessian(energy(P)), in_dims=(0, None)), in_dims=(0, 0))(F, pe)      # (n_el, n_q, 2, 2, 2, 2)
    n_el, n_q = F.shape[:2]
    return (H * P["w_detJ"][:, :, None, None, None, None]).reshape(n_el, n_q, 4, 4)


def apply_qp(C, v, P):
    """A(v) with a batched 4x4 matmul per Gauss point (make_A_operator_qp, operators.py:373-380)."""
    m, conn, dN = P["m"], P["conn"], P["dN_dX"]
    n_el, n_q = C.shape[:2]
    ve = gather_nodes(m * v, conn)
    dgrad = torch.einsum("eai,eqaj->eqij", ve, dN).reshape(n_el, n_q, 4, 1)
    dP = torch.matmul(C, dgrad).reshape(n_el, n_q, 2, 2)
    fe = torch.einsum("eqij,eqaj->eai", dP, dN)
    return m * scatter_nodes(fe, conn, P["nodes"].shape[0]) + (1.0 - m) * v


def apply_qp_ew(C, v, P):
    """A(v) as broadcast multiply + sum (make_A_operator_qp_ew, operators.py:403-410): the FP64 oracle."""
    m, conn, dN = P["m"], P["conn"], P["dN_dX"]
    n_el, n_q = C.shape[:2]
    ve = gather_nodes(m * v, conn)
    dgrad = (ve[:, None, :, :, None] * dN[:, :, :, None, :]).sum(2)
    dP = (C * dgrad.reshape(n_el, n_q, 1, 4)).sum(-1).reshape(n_el, n_q, 2, 2)
    fe = (dP[:, :, None, :, :] * dN[:, :, :, None, :]).sum(dim=(1, 4))
    return m * scatter_nodes(fe, conn, P["nodes"].shape[0]) + (1.0 - m) * v


def make_operator(kind, u, theta, P):
    """v -> A(v): "qp" / "qp_ew" store the moduli once; "jvp" differentiates the residual (operators.py:231-275)."""
    if kind == "jvp":
        m = P["m"]

        def A(v):
            _, Jv = jvp(lambda w: residual(w, theta, P), (u,), (m * v,))
            return m * Jv + (1.0 - m) * v
        return A
    C = moduli(u, theta, P)
    if kind == "qp":
        return lambda v: apply_qp(C, v, P)
    if kind == "qp_ew":
        return lambda v: apply_qp_ew(C, v, P)
    raise ValueError(kind)


def make_transpose_operator(u, theta, P):
    """v -> m J^T (m v) + (1 - m) v by reverse-mode AD (make_AT_operator, operators.py:441-471)."""
    m = P["m"]
    _, pullback = vjp(lambda w: residual(w, theta, P), u)

    def AT(v):
        (JTv,) = pullback(m * v)
        return m * JTv + (1.0 - m) * v
    return AT


# ---------------------------------------------------------------------------------------------
# Jacobi diagonal (operators.py:477-570)
# ---------------------------------------------------------------------------------------------
def jacobi_diagonal(u, theta, P):
    """diag(K) from one jvp of the element force per local unit vector, clamped and pivoted."""
    conn, dN, wd = P["conn"], P["dN_dX"], P["w_detJ"]
    n_el, nen = conn.shape
    ue = gather_nodes(u, conn)
    pe = element_parameters(theta, P)
    psi_e = energy(P)
    basis = torch.eye(2 * nen, dtype=F64).reshape(2 * nen, nen, 2)

    def force(w, dN_e, wd_e, p_e):
        F = torch.eye(2, dtype=F64) + torch.einsum("ai,qaj->qij", w, dN_e)
        st = vmap(grad(psi_e), in_dims=(0, None))(F, p_e)
        return torch.einsum("q,qij,qaj->ai", wd_e, st, dN_e)

    def entry(u_e, dN_e, wd_e, p_e, e_vec):
        _, t = jvp(lambda w: force(w, dN_e, wd_e, p_e), (u_e,), (e_vec,))
        return (t * e_vec).sum()

    per_el = vmap(lambda a, b, c, d: vmap(entry, in_dims=(None, None, None, None, 0))(a, b, c, d, basis))(
        ue, dN, wd, pe)
    diag = scatter_nodes(per_el.reshape(n_el, nen, 2), conn, P["nodes"].shape[0])
    return torch.where(P["m"] > 0.0, torch.clamp(diag, min=1e-6), torch.ones_like(diag))


def block_jacobi(u, theta, P):
    """
    Nodal block-Jacobi M^-1 (operators.py:586-625): the 2x2 diagonal block of every element tangent from
    one jvp of the element force per local unit vector (its node's rows), scattered to the nodes, identity
    rows/columns on fixed DOFs, + 1e-12 I, inverted.  Returns the closure r -> Binv r.
    """
    conn, dN, wd = P["conn"], P["dN_dX"], P["w_detJ"]
    n_el, nen = conn.shape
    N = P["nodes"].shape[0]
    ue = gather_nodes(u, conn)
    pe = element_parameters(theta, P)
    psi_e = energy(P)
    basis = torch.eye(2 * nen, dtype=F64).reshape(2 * nen, nen, 2)
    node_of = torch.arange(2 * nen) // 2

    def force(w, dN_e, wd_e, p_e):
        F = torch.eye(2, dtype=F64) + torch.einsum("ai,qaj->qij", w, dN_e)
        st = vmap(grad(psi_e), in_dims=(0, None))(F, p_e)
        return torch.einsum("q,qij,qaj->ai", wd_e, st, dN_e)

    def column(u_e, dN_e, wd_e, p_e, e_vec, a):
        _, t = jvp(lambda w: force(w, dN_e, wd_e, p_e), (u_e,), (e_vec,))
        return t[a]                                             # rows of node a: column j of its block

    cols = vmap(lambda a, b, c, d: vmap(column, in_dims=(None, None, None, None, 0, 0))(a, b, c, d, basis, node_of))(
        ue, dN, wd, pe)                                         # (n_el, 2 nen, 2): [e, (a, j), i]
    blocks = cols.reshape(n_el, nen, 2, 2).transpose(2, 3)      # [e, a, i, j]
    B = torch.zeros(N, 2, 2, dtype=F64).index_add_(0, conn.reshape(-1), blocks.reshape(-1, 2, 2))
    mn = P["m"].reshape(N, 2)
    B = B * (mn[:, :, None] * mn[:, None, :]) + torch.diag_embed(1.0 - mn) + 1e-12 * torch.eye(2, dtype=F64)
    Binv = torch.linalg.inv(B)
    return lambda r: torch.einsum("nij,nj->ni", Binv, r.reshape(N, 2)).reshape(-1)


def assemble_tangent(u, theta, P):
    """
    The tangent as a SciPy CSC matrix with identity pivots on constrained DOFs (assemble_tangent_sparse,
    operators.py:641-677).  The element matrices K_e[(a i), (b k)] = sum_q sum_JL dN_aJ C_(iJ)(kL) dN_bL come
    from the stored moduli (the same second derivatives the reference takes by jacfwd of the element force),
    scattered once as COO entries with the rows and columns of constrained DOFs dropped.
    """
    import numpy as np
    import scipy.sparse as sp
    conn, m, dN = P["conn"], P["m"], P["dN_dX"]
    n_el, nen = conn.shape
    C = moduli(u, theta, P).reshape(n_el, -1, 2, 2, 2, 2)                     # [e, q, i, J, k, L]
    Ke = torch.einsum("eqaJ,eqiJkL,eqbL->eaibk", dN, C, dN).reshape(n_el, 2 * nen, 2 * nen)
    dofs = (2 * conn[:, :, None] + torch.arange(2)).reshape(n_el, 2 * nen)
    rows = dofs[:, :, None].expand(-1, -1, 2 * nen).reshape(-1)
    cols = dofs[:, None, :].expand(-1, 2 * nen, -1).reshape(-1)
    free = m > 0.5
    vals = Ke.reshape(-1) * (free[rows] & free[cols])
    fixed_ids = torch.nonzero(~free).reshape(-1)
    rows = torch.cat([rows, fixed_ids]).numpy()
    cols = torch.cat([cols, fixed_ids]).numpy()
    vals = torch.cat([vals, torch.ones(fixed_ids.numel(), dtype=F64)]).numpy()
    n = m.numel()
    return sp.coo_matrix((vals, (rows, cols)), shape=(n, n)).tocsc().astype(np.float64)


def ilu_preconditioner(u, theta, P, drop_tol=1e-5, fill_factor=30.0):
    """Incomplete LU of the assembled tangent, SciPy spilu (make_ilu_preconditioner, operators.py:680-699)."""
    from scipy.sparse.linalg import spilu
    ilu = spilu(assemble_tangent(u, theta, P), drop_tol=drop_tol, fill_factor=fill_factor)
    return lambda r: torch.as_tensor(ilu.solve(r.numpy()), dtype=F64)


def preconditioner(kind, u, theta, P):
    """M^-1 as a closure: "jacobi" (r / diag), "block_jacobi" or "ilu" (operators.py:702-710)."""
    if kind == "jacobi":
        d = jacobi_diagonal(u, theta, P)
        return lambda r: r / d
    if kind == "block_jacobi":
        return block_jacobi(u, theta, P)
    if kind == "ilu":
        return ilu_preconditioner(u, theta, P)
    raise ValueError(kind)


# ---------------------------------------------------------------------------------------------
# PCG, line search, Newton, continuation (newton_krylov.py:28-274)
# ---------------------------------------------------------------------------------------------
def pcg(A, b, Minv, rtol=1e-5, max_iter=500):
    """Textbook PCG with x0 = 0 (newton_krylov.py:28-88): returns (x, iterations)."""
    x = torch.zeros_like(b)
    r = b.clone()
    z = Minv(r)
    p = z.clone()
    rz = torch.dot(r, z)
    nb = torch.norm(b)
    if nb == 0.0:
        return x, 0
    for k in range(max_iter):
        Ap = A(p)
        curv = torch.dot(p, Ap)
        if curv <= 0.0:
            return (z if k == 0 else x), k
        a = rz / curv
        x = x + a * p
        r = r - a * Ap
        if torch.norm(r) <= rtol * nb:
            return x, k + 1
        z = Minv(r)
        rz_next = torch.dot(r, z)
        p = z + (rz_next / rz) * p
        rz = rz_next
    return x, max_iter


def line_search(u, du, rn, theta, P, lf, c1=1e-4, min_alpha=2.0 ** -5):
    """Armijo backtracking on ||R|| (newton_krylov.py:94-120)."""
    alpha = 1.0
    while alpha >= min_alpha:
        uc = u + alpha * du
        Rc = residual(uc, theta, P, lf)
        rc = torch.norm(Rc)
        if rc < (1.0 - c1 * alpha) * rn:
            return uc, Rc, rc, alpha, True
        alpha *= 0.5
    return u, None, rn, alpha, False


def newton_at_load(u0, theta, P, lf, tol, max_newton, tangent="qp", pcg_max_iter=500, precond="jacobi"):
    """Inexact Newton with the Eisenstat-Walker forcing term (newton_krylov.py:126-179)."""
    u = torch.where(P["fixed"], lf * P["u_D"], u0)
    R = residual(u, theta, P, lf)
    r0 = rn = torch.norm(R)
    records = []
    for it in range(max_newton + 1):
        if rn < tol:
            return u, True, records
        if it == max_newton:
            break
        eta = min(0.5, float((rn / (r0 + 1e-14)) ** 0.5))
        A = make_operator(tangent, u, theta, P)
        du, iters = pcg(A, -R, preconditioner(precond, u, theta, P), rtol=eta, max_iter=pcg_max_iter)
        u, R_new, rn, alpha, ok = line_search(u, du, rn, theta, P, lf)
        records.append(dict(iteration=it, residual=float(rn), cg_iters=int(iters), alpha=alpha, load_factor=lf))
        if not ok:
            return u, False, records
        R = R_new
    return u, False, records


@torch.no_grad()
def newton_krylov_solve(P, theta, n_load_steps=5, tol=1e-8, max_newton=25, max_cutbacks=8, tangent="qp",
                        pcg_max_iter=500, precond="jacobi"):
    """Load continuation with cut-backs (newton_krylov.py:185-264); returns (u, info)."""
    u = torch.zeros(2 * P["nodes"].shape[0], dtype=F64)
    info = dict(converged=False, load_factor=0.0, history=[], total_newton=0, total_cg=0, n_cutbacks=0)
    d_nom = 1.0 / n_load_steps
    d_lf, lf, streak = d_nom, 0.0, 0
    while lf < 1.0 - 1e-12:
        lf_try = min(1.0, lf + d_lf)
        u_try, ok, rec = newton_at_load(u, theta, P, lf_try, tol, max_newton, tangent, pcg_max_iter, precond)
        info["history"] += rec
        info["total_newton"] += len(rec)
        info["total_cg"] += sum(r["cg_iters"] for r in rec)
        if ok:
            u, lf, streak = u_try, lf_try, 0
            d_lf = min(d_nom, 1.5 * d_lf)
        else:
            streak += 1
            info["n_cutbacks"] += 1
            if streak > max_cutbacks:
                info["load_factor"] = lf
                return u, info
            d_lf *= 0.5
    info["converged"], info["load_factor"] = True, 1.0
    return u, info


# ---------------------------------------------------------------------------------------------
# adjoint sensitivities (adjoint.py:31-106, sensitivity.py:7-38)
# ---------------------------------------------------------------------------------------------
def solve_adjoint(u, theta, P, dL_du, rtol=1e-6, max_iter=500):
    """A^T lambda = m dL/du by Jacobi-PCG with the vjp transpose operator (adjoint.py:31-69)."""
    AT = make_transpose_operator(u, theta, P)
    d = jacobi_diagonal(u, theta, P)
    return pcg(AT, P["m"] * dL_du, lambda r: r / d, rtol=rtol, max_iter=max_iter)


def implicit_vjp(u, theta, P, lam):
    """dL/dtheta = -lambda^T dR/dtheta by one vjp w.r.t. theta at load factor 1 (adjoint.py:75-106)."""
    _, pullback = vjp(lambda th: residual(u, th, P, 1.0), theta)
    (g,) = pullback(-lam)
    return g


def compute_sensitivity(P, theta, loss_fn, n_load_steps=5, tol=1e-8, max_newton=25, adjoint_rtol=1e-10,
                        adjoint_max_iter=500, pcg_max_iter=500):
    """(u*, dL/dtheta) (sensitivity.py:7-38)."""
    u, _ = newton_krylov_solve(P, theta, n_load_steps, tol, max_newton, pcg_max_iter=pcg_max_iter)
    dL_du = grad(loss_fn)(u)
    lam, _ = solve_adjoint(u, theta, P, dL_du, rtol=adjoint_rtol, max_iter=adjoint_max_iter)
    return u, implicit_vjp(u, theta, P, lam)


# ---------------------------------------------------------------------------------------------
# post-processing (postprocess.py:24-137)
# ---------------------------------------------------------------------------------------------
def gauss_point_state(F, p, psi3):
    """[J, sxx, syy, sxy, szz, psi] at one Gauss point: P3 = d psi3 / d F3, sigma = P3 F3^T / J (postprocess.py:24-47)."""
    F3 = torch.cat([torch.cat([F, torch.zeros(2, 1, dtype=F.dtype)], 1),
                    torch.tensor([[0.0, 0.0, 1.0]], dtype=F.dtype)], 0)
    P3 = grad(psi3)(F3, p)
    J = F[0, 0] * F[1, 1] - F[0, 1] * F[1, 0]
    sigma = P3 @ F3.T / J
    return torch.stack([J, sigma[0, 0], sigma[1, 1], sigma[0, 1], sigma[2, 2], psi3(F3, p)])


def compute_fields(u, theta, P):
    """compute_fields (postprocess.py:70-118): w detJ-weighted element means, von Mises, nodal averages."""
    conn, N = P["conn"], P["nodes"].shape[0]
    F = deformation_gradient(gather_nodes(u, conn), P["dN_dX"])
    pe = element_parameters(theta, P)
    psi3 = PSI3[P.get("material", "neo_hookean")]
    S = vmap(vmap(lambda F_, p_: gauss_point_state(F_, p_, psi3), in_dims=(0, None)), in_dims=(0, 0))(F, pe)
    w = P["w_detJ"]
    area = w.sum(1)
    mean = torch.einsum("eq,eqk->ek", w, S) / area[:, None]
    J, sxx, syy, sxy, szz, dens = mean.unbind(1)
    mises = torch.sqrt(0.5 * ((sxx - syy) ** 2 + (syy - szz) ** 2 + (szz - sxx) ** 2) + 3.0 * sxy ** 2)
    un = u.reshape(N, 2)
    out = {"J": J, "sxx": sxx, "syy": syy, "sxy": sxy, "mises": mises, "energy_density": dens,
           "ux": un[:, 0], "uy": un[:, 1], "u_mag": torch.linalg.norm(un, dim=1),
           "strain_energy": torch.sum(dens * area), "min_J": J.min()}
    for name in ("ux", "uy", "u_mag"):
        out[name + "_n"] = out[name]
    count = torch.zeros(N, dtype=F64).index_add_(0, conn.reshape(-1), torch.ones(conn.numel(), dtype=F64))
    for name in ("J", "sxx", "syy", "sxy", "mises", "energy_density"):
        s = torch.zeros(N, dtype=F64).index_add_(0, conn.reshape(-1), out[name][:, None].expand(-1, conn.shape[1]).reshape(-1))
        out[name + "_n"] = s / count.clamp(min=1.0)
    return out


def support_reactions(u, theta, P):
    """Total (Rx, Ry) of the unmasked internal force over the fixed DOFs (postprocess.py:121-137)."""
    R = scatter_nodes(element_forces(u, theta, P), P["conn"], P["nodes"].shape[0]).reshape(-1, 2)
    fixed = P["fixed"].reshape(-1, 2)
    return torch.sum(torch.where(fixed, R, torch.zeros_like(R)), dim=0)
