"""
Newton-Krylov solver on the GPU (the reference's newton_krylov.py API and semantics).

    pcg(A_fn, b, Minv_fn, rtol=1e-5, max_iter=500)                       newton_krylov.py:28-88
    armijo_line_search(u, du, rn, theta, params, load_factor, ...)        newton_krylov.py:94-120
    newton_at_load(u0, theta, params, load_factor, tol, max_newton, ...)  newton_krylov.py:126-179
    newton_krylov_solve(params, theta, n_load_steps=5, tol=1e-8, ...)     newton_krylov.py:185-264
    solve_newton_krylov(...)                                              newton_krylov.py:267-274

The control flow is the reference's: load continuation with cut-backs (halve the increment on failure,
up to ``max_cutbacks`` in a row, grow it by 1.5 after a success), inexact Newton with the forcing term
eta = min(0.5, sqrt(||R|| / ||R_0||)), Jacobi-PCG capped at ``pcg_max_iter`` (500 in the reference),
Armijo backtracking from alpha = 1 down to 2^-5 with c1 = 1e-4, NaN (inverted element) rejecting a step.
What changes is where it runs: the residual (with its norm), the moduli and diagonal, and the whole PCG
are device kernels on buffers held by a ``NewtonWorkspace``; the host reads back one scalar per residual
and (status, iterations) per linear solve.

``preconditioner`` is "jacobi" (the reference's default) or "block_jacobi" (nodal 2x2 blocks,
operators.py:586-625), both applied inside the device PCG.

Extra keyword arguments (not in the reference): ``pcg_max_iter``; ``precision`` = "fp64" (default) or
"fp32" (the PCG applies FP32 moduli and gradients -- the bytes that dominate the operator -- to FP64
Krylov vectors; the residual, line search, convergence test and state update stay FP64, so each Newton
step is an iterative-refinement correction of the FP64 state computed with an FP32 operator);
``workspace`` to reuse device buffers across solves of the same problem.
"""
import torch

from difffea_b200.operators import (CudaBlockJacobiPreconditioner, CudaJacobiPreconditioner, CudaTangentOperator,
                                    PRECONDITIONERS, REFERENCE_TANGENT_VARIANTS, TANGENT_OPERATORS)
from difffea_b200.workspace import NewtonWorkspace

# inner-solve floor with the FP32 operator: the solve is of the operator rounded to FP32, so asking it
# for more than a few digits beyond kappa * eps_32 buys nothing for the Newton step
FP32_MIN_RTOL = 1e-5


# =============================================================================================
# PCG
# =============================================================================================
def pcg(A_fn, b, Minv_fn, rtol=1e-5, max_iter=500):
    """
    Solve A x = b by preconditioned CG with x0 = 0; returns (x, iterations).

    Stops when ||r|| <= rtol ||b||, returns (0, 0) for b = 0, and on non-positive curvature p.Ap <= 0
    returns z = M^-1 b at the first iteration and the current x otherwise.  With the GPU operator and
    Jacobi preconditioner of this package the whole loop runs on the device (kernel (c), one CUDA
    graph); any other pair of closures runs the same recurrences step by step.
    """
    if (isinstance(A_fn, CudaTangentOperator) and isinstance(Minv_fn, CudaJacobiPreconditioner)
            and Minv_fn.mesh is A_fn.mesh and b.is_cuda):
        return A_fn.pcg_solve(b, Minv_fn.diag, rtol, max_iter)
    if (isinstance(A_fn, CudaTangentOperator) and isinstance(Minv_fn, CudaBlockJacobiPreconditioner)
            and Minv_fn.mesh is A_fn.mesh and b.is_cuda):
        return A_fn.pcg_solve(b, Minv_fn.blocks, rtol, max_iter, preconditioner="block_jacobi")
    return _pcg_steps(A_fn, b, Minv_fn, rtol, max_iter)


def _pcg_steps(A_fn, b, Minv_fn, rtol, max_iter):
    """Textbook PCG (Saad, Alg. 9.1) on arbitrary closures, one host decision per iteration."""
    x = torch.zeros_like(b)
    r = b.clone()
    z = Minv_fn(r)
    p = z.clone()
    rz = torch.dot(r, z)
    norm_b = torch.norm(b)
    if norm_b == 0.0:
        return x, 0
    for k in range(max_iter):
        Ap = A_fn(p)
        curv = torch.dot(p, Ap)
        if curv <= 0.0:
            return (z if k == 0 else x), k
        alpha = rz / curv
        x = x + alpha * p
        r = r - alpha * Ap
        if torch.norm(r) <= rtol * norm_b:
            return x, k + 1
        z = Minv_fn(r)
        rz_new = torch.dot(r, z)
        p = z + (rz_new / rz) * p
        rz = rz_new
    return x, max_iter


# =============================================================================================
# line search, Newton, continuation
# =============================================================================================
def _check_kinds(tangent, preconditioner):
    if tangent not in TANGENT_OPERATORS:
        if tangent in REFERENCE_TANGENT_VARIANTS:
            raise ValueError(f"tangent '{tangent}' is one of the reference's PyTorch variants; "
                             f"difffea_b200 provides {TANGENT_OPERATORS}")
        raise ValueError(f"Unknown tangent operator '{tangent}'. Choose one of {TANGENT_OPERATORS}.")
    if preconditioner not in PRECONDITIONERS:
        raise ValueError(f"Unknown preconditioner '{preconditioner}'. Choose one of {PRECONDITIONERS}.")


def _workspace(params, theta, precision, workspace, preconditioner="jacobi"):
    ws = workspace if workspace is not None else NewtonWorkspace(params, precision, preconditioner=preconditioner)
    if ws.precision != precision:
        raise ValueError("workspace precision does not match")
    if ws.preconditioner != preconditioner:
        raise ValueError(f"workspace preconditioner '{ws.preconditioner}' does not match '{preconditioner}'")
    ws.set_theta(theta)
    return ws


def armijo_line_search(u, du, rn, theta, params, load_factor, c1=1e-4, min_alpha=2.0 ** -5, *, workspace=None,
                       precision="fp64", preconditioner="jacobi"):
    """
    Backtrack alpha = 1, 1/2, ... >= min_alpha until ||R(u + alpha du)|| < (1 - c1 alpha) ||R(u)||.
    Returns (u_new, R_new, ||R_new||, alpha, accepted); (u, None, rn, alpha, False) if no step passes.
    """
    ws = _workspace(params, theta, precision, workspace, preconditioner)
    rn = float(rn)
    alpha = 1.0
    while alpha >= min_alpha:
        uc = ws.trial(u, alpha, du, torch.empty_like(u))
        rn_c = ws.residual(uc, load_factor, ws.Rc)
        if rn_c < (1.0 - c1 * alpha) * rn:        # False for NaN: an inverted element rejects the step
            ws.R, ws.Rc = ws.Rc, ws.R
            return uc, ws.R, rn_c, alpha, True
        alpha *= 0.5
    return u, None, rn, alpha, False


def newton_at_load(u0, theta, params, load_factor, tol, max_newton, verbose, callback, step_id,
                   preconditioner="jacobi", tangent="auto", *, pcg_max_iter=500, precision="fp64", workspace=None):
    """Inexact Newton-Krylov at one load factor; returns (u, converged, records)."""
    _check_kinds(tangent, preconditioner)
    ws = _workspace(params, theta, precision, workspace, preconditioner)
    u = torch.where(params["fixed"], load_factor * params["u_D"], u0).to(torch.float64).contiguous()
    rn = ws.residual(u, load_factor, ws.R)
    r0 = rn
    records = []
    for it in range(max_newton + 1):
        if rn < tol:
            if verbose:
                print(f"  converged in {it} Newton iterations (||R|| = {rn:.3e})")
            return u, True, records
        if it == max_newton:
            break
        eta = min(0.5, float((rn / (r0 + 1e-14)) ** 0.5))
        rtol = max(eta, FP32_MIN_RTOL) if precision == "fp32" else eta
        ws.linearize(u)
        du, cg_iters, _ = ws.solve(ws.R, rtol, pcg_max_iter)
        u, R_new, rn, alpha, accepted = armijo_line_search(u, du, rn, theta, params, load_factor, workspace=ws,
                                                           precision=precision, preconditioner=preconditioner)
        record = dict(step=step_id, load_factor=load_factor, iteration=it, residual=float(rn),
                      cg_iters=int(cg_iters), alpha=alpha)
        records.append(record)
        if callback is not None:
            callback(record)
        if verbose:
            print(f"  iter {it:2d} | ||R|| = {rn:.4e} | CG = {cg_iters:3d} | alpha = {alpha:.4f}")
        if not accepted:
            return u, False, records
    return u, False, records


@torch.no_grad()
def newton_krylov_solve(params, theta, n_load_steps=5, tol=1e-8, max_newton=25, verbose=True, callback=None,
                        max_cutbacks=8, preconditioner="jacobi", tangent="auto", *, pcg_max_iter=500,
                        precision="fp64", workspace=None, driver="python"):
    """
    Solve R(u, theta) = 0 with load continuation; returns (u, info) with info keys converged,
    load_factor, history, total_newton, total_cg, n_cutbacks, snapshots (as the reference).

    ``driver``: "python" runs the loop here (per-step callback, verbose printing, a snapshot per load step);
    "native" runs the same loop in the library's C++ driver (dfea_newton_solve), the same iterates bit for
    bit, in one call that holds no interpreter lock -- for many solves on concurrent host threads.  It takes
    no callback, prints the history after the solve when verbose, and keeps the initial and final
    snapshots only.
    """
    _check_kinds(tangent, preconditioner)
    nodes = params["nodes"]
    if not nodes.is_cuda:
        raise RuntimeError("difffea_b200 solves on CUDA devices only: move the problem with "
                           "problem.to_device(params, 'cuda')")
    if driver not in ("python", "native"):
        raise ValueError("driver must be 'python' or 'native'")
    ws = _workspace(params, theta, precision, workspace, preconditioner)
    if driver == "native":
        if callback is not None:
            raise ValueError("the native driver takes no callback (use driver='python')")
        u, info = ws.native_solve(theta, n_load_steps, tol, max_newton=max_newton, max_cutbacks=max_cutbacks,
                                  pcg_max_iter=pcg_max_iter)
        if verbose:
            for r in info["history"]:
                print(f"  step {r['step']} iter {r['iteration']:2d} | ||R|| = {r['residual']:.4e} | "
                      f"CG = {r['cg_iters']:3d} | alpha = {r['alpha']:.4f}")
        return u, info
    u = torch.zeros(2 * nodes.shape[0], dtype=torch.float64, device=nodes.device)
    info = {"converged": False, "load_factor": 0.0, "history": [], "total_newton": 0, "total_cg": 0,
            "n_cutbacks": 0, "snapshots": [(0.0, u.clone())]}
    d_nominal = 1.0 / n_load_steps
    d_lf, lf = d_nominal, 0.0
    step_id, cutbacks_in_row = 0, 0
    while lf < 1.0 - 1e-12:
        lf_try = min(1.0, lf + d_lf)
        step_id += 1
        if verbose:
            print(f"\n=== Load step {step_id}: load factor {lf:.3f} -> {lf_try:.3f} ===")
        u_try, ok, records = newton_at_load(u, theta, params, lf_try, tol, max_newton, verbose, callback, step_id,
                                            preconditioner, tangent, pcg_max_iter=pcg_max_iter, precision=precision,
                                            workspace=ws)
        info["history"] += records
        info["total_newton"] += len(records)
        info["total_cg"] += sum(r["cg_iters"] for r in records)
        if ok:
            u, lf = u_try, lf_try
            info["snapshots"].append((lf, u.clone()))
            cutbacks_in_row = 0
            d_lf = min(d_nominal, 1.5 * d_lf)
        else:
            cutbacks_in_row += 1
            info["n_cutbacks"] += 1
            if cutbacks_in_row > max_cutbacks:
                info["load_factor"] = lf
                return u, info
            d_lf *= 0.5
            if verbose:
                print(f"  Newton failed -> load increment reduced to {d_lf:.4f}")
    info["converged"] = True
    info["load_factor"] = 1.0
    return u, info


def solve_newton_krylov(params, theta, n_load_steps=5, tol=1e-8, max_newton=25, verbose=True, **kw):
    """``newton_krylov_solve`` returning only u."""
    u, _ = newton_krylov_solve(params, theta, n_load_steps=n_load_steps, tol=tol, max_newton=max_newton,
                               verbose=verbose, **kw)
    return u
