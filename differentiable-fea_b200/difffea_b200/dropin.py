"""
Register the "cuda" tangent variant inside an installed difffea package, at run time.

The reference selects its tangent operator and preconditioner by name inside its own Newton loop
(newton_krylov.py:160-164 calls make_tangent_operator(tangent, ...) and make_preconditioner(preconditioner,
...), then pcg(A_fn, -R, Minv_fn, rtol=eta)).  A maintainer adds the variant to its source (the lines of
operators.py:415-435 / 702-710 and newton_krylov.py:28); ``register`` applies the same change to the imported
modules, for a user who cannot edit the installed package:

    import difffea
    from difffea_b200.dropin import register
    undo = register(difffea)
    u, info = difffea.newton_krylov.newton_krylov_solve(params_cuda, theta, tangent="cuda")
    undo()                                   # the package as it was

After ``register`` the reference's names behave as follows; every other name keeps its own behaviour:

    TANGENT_OPERATORS       gains "cuda"
    make_tangent_operator   "cuda" -> difffea_b200's stored-moduli operator (kernels (a), (b)); other names
                            go to the reference's own variants
    PRECONDITIONERS         gains "multigrid"
    make_preconditioner     "jacobi" with a CUDA state -> the diagonal from kernel (a); "multigrid" -> the
                            geometric multigrid V-cycle of a structured mesh; other cases go to the reference
    pcg                     the cuda operator with its Jacobi preconditioner -> the device-resident PCG (one
                            CUDA graph per solve); with the multigrid preconditioner -> the device PCG driven
                            from C++; any other pair -> the reference's own PCG loop

The reference's Newton loop, line search, load continuation and residual run unchanged, so its own
``newton_krylov_solve(..., tangent="cuda")`` drives the kernels of this package.
"""
import importlib

import torch

_PATCHED = "_difffea_b200_registered"


def _modules(package):
    if package is None:
        package = importlib.import_module("difffea")
    name = package if isinstance(package, str) else package.__name__
    return importlib.import_module(name + ".operators"), importlib.import_module(name + ".newton_krylov")


def register(package=None):
    """
    Add the "cuda" variant (and the "multigrid" preconditioner) to difffea's operator and PCG dispatch.
    ``package`` is the imported difffea package (or its name; default "difffea").  Returns a function that
    restores the original names.  Registering twice is a no-op that returns the first undo function.
    """
    from difffea_b200.operators import (CudaJacobiPreconditioner, CudaMultigridPreconditioner, CudaTangentOperator,
                                        make_A_operator_cuda, make_jacobi_preconditioner,
                                        make_multigrid_preconditioner)
    ops, nk = _modules(package)
    if getattr(ops, _PATCHED, None) is not None:
        return getattr(ops, _PATCHED)

    saved = {(m, k): getattr(m, k) for m in (ops, nk)
             for k in ("make_tangent_operator", "make_preconditioner", "pcg", "TANGENT_OPERATORS", "PRECONDITIONERS")
             if hasattr(m, k)}
    ref_tangent, ref_pre, ref_pcg = ops.make_tangent_operator, ops.make_preconditioner, nk.pcg

    def make_tangent_operator(kind, u, theta, params):
        if kind == "cuda":
            return make_A_operator_cuda(u, theta, params)
        return ref_tangent(kind, u, theta, params)

    def make_preconditioner(kind, u, theta, params):
        if kind == "jacobi" and u.is_cuda:
            return make_jacobi_preconditioner(u, theta, params)
        if kind == "multigrid":
            return make_multigrid_preconditioner(u, theta, params)
        return ref_pre(kind, u, theta, params)

    def pcg(A_fn, b, Minv_fn, rtol=1e-5, max_iter=500):
        if isinstance(A_fn, CudaTangentOperator) and b.is_cuda:
            if isinstance(Minv_fn, CudaJacobiPreconditioner) and Minv_fn.mesh is A_fn.mesh:
                return A_fn.pcg_solve(b, Minv_fn.diag, rtol, max_iter)
            if isinstance(Minv_fn, CudaMultigridPreconditioner) and Minv_fn.mesh is A_fn.mesh:
                Minv_fn.refresh()                       # the hierarchy at this closure's linearisation
                x = torch.empty_like(b, dtype=torch.float64)
                iters, _ = Minv_fn.mg.pcg(b.to(torch.float64).contiguous(), x, rtol, max_iter)
                return x.to(b.dtype), iters
        return ref_pcg(A_fn, b, Minv_fn, rtol=rtol, max_iter=max_iter)

    tangents = tuple(ops.TANGENT_OPERATORS) + ("cuda",)
    preconditioners = tuple(getattr(ops, "PRECONDITIONERS", ())) + ("multigrid",)
    for m in (ops, nk):
        for k, v in (("make_tangent_operator", make_tangent_operator), ("make_preconditioner", make_preconditioner),
                     ("pcg", pcg)):
            if (m, k) in saved:
                setattr(m, k, v)
        if (m, "TANGENT_OPERATORS") in saved:
            m.TANGENT_OPERATORS = tangents
        if (m, "PRECONDITIONERS") in saved:
            m.PRECONDITIONERS = preconditioners

    def undo():
        for (m, k), v in saved.items():
            setattr(m, k, v)
        if hasattr(ops, _PATCHED):
            delattr(ops, _PATCHED)

    setattr(ops, _PATCHED, undo)
    return undo
