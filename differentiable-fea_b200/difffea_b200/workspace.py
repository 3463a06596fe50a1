"""
Per-problem device workspace of the Newton-Krylov solver.

A ``NewtonWorkspace`` keeps everything a solve touches in HBM for the whole solve: the state and
trial vectors, the residual, the Gauss-point moduli (FP64, or for the mixed-precision form FP32 moduli
pulled back to each element's reference frame, so that its operator reads 10 FP32 numbers per Gauss
point and no gradients, while the Krylov vectors stay FP64), the Jacobi diagonal,
and one graph-captured ``DevicePCG`` bound to them (eight iterations per graph launch, replayed until
the solve ends: faster than the conditional-loop graph, 23 vs 28 us per iteration at 16k elements).  The solver loop
calls the C ABI directly on these buffers (no allocation per Newton step), reading back only the
scalars the algorithm branches on: ||R|| per residual evaluation and (status, iterations) per PCG.
"""
import torch

from difffea_b200 import _lib
from difffea_b200.cuda_mesh import _require_cuda, cuda_mesh, ptr, stream_handle
from difffea_b200.krylov import DevicePCG
from difffea_b200.materials import device_material


# Below this many elements the fused gather form of the PCG iteration (2 kernels) is faster than the
# colour form (n_colours + 2 kernels); above it the colour form's lower traffic wins (measured on B200,
# FP64, per iteration: 23.0 vs 40.2 us at 16k Q4 elements, 27.5 vs 46.5 at 40k, 171 vs 174 at 640k,
# 608 vs 550 at 2.56M).
GATHER_FORM_MAX_ELEMENTS = 1_500_000


def pcg_form_for(mesh, pcg_form="auto"):
    """The PCG product form: "colour", "gather", "fused", or "auto" (fused below GATHER_FORM_MAX_ELEMENTS)."""
    if pcg_form == "auto":
        return "fused" if mesh.n_el < GATHER_FORM_MAX_ELEMENTS else "colour"
    if pcg_form not in ("colour", "gather", "fused"):
        raise ValueError("pcg_form must be 'auto', 'colour', 'gather' or 'fused'")
    return pcg_form


class NewtonWorkspace:
    def __init__(self, params, precision="fp64", use_graph=2, pcg_form="auto", fp32_moduli="ref", max_blocks=0,
                 preconditioner="jacobi", batch=None):
        if precision not in ("fp64", "fp32"):
            raise ValueError("precision must be 'fp64' or 'fp32' (FP32 moduli and PCG, FP64 Newton)")
        if preconditioner not in ("jacobi", "block_jacobi", "multigrid"):
            raise ValueError("preconditioner must be 'jacobi', 'block_jacobi' or 'multigrid'")
        self.preconditioner = preconditioner
        self.params = params
        self.mesh = mesh = cuda_mesh(params)
        self.material = device_material(params)
        self.precision = precision
        dev, n = mesh.device, mesh.n_dof
        f64 = dict(dtype=torch.float64, device=dev)
        self.f = params["f"].detach().to(**f64).contiguous()
        self.R = torch.empty(n, **f64)
        self.Rc = torch.empty(n, **f64)
        self.uc = torch.empty(n, **f64)
        self.du = torch.empty(n, **f64)
        self.diag = torch.empty(n, **f64)
        # block-Jacobi: the inverse 2x2 node blocks (Binv00, Binv01, Binv11, 0) per node
        self.blocks = torch.empty(2 * n, **f64) if preconditioner == "block_jacobi" else None
        self.scal = torch.zeros(4, **f64)
        self.scal_host = torch.zeros(4, dtype=torch.float64).pin_memory()
        # "fp32": the operator's bytes in FP32, Krylov vectors and scalars in FP64.  fp32_moduli "ref":
        # moduli pulled back to the element reference frame, 10 per Gauss point, no gradients read
        # (the default); "physical": the 16 moduli with FP32 gradients.
        if fp32_moduli not in ("ref", "physical"):
            raise ValueError("fp32_moduli must be 'ref' or 'physical'")
        self.moduli_kind = "ref" if (precision == "fp32" and fp32_moduli == "ref") else "physical"
        if self.moduli_kind == "ref":
            mesh.ensure_ref_frame()
            self.C = torch.empty(mesh.moduli_numel_ref(), dtype=torch.float32, device=dev)
            self.moduli_code = _lib.DFEA_F32REF
        else:
            self.C = torch.empty(mesh.moduli_numel(), dtype=torch.float64 if precision == "fp64" else torch.float32,
                                 device=dev)
            self.moduli_code = _lib.DFEA_F64 if precision == "fp64" else _lib.DFEA_F32
            if precision == "fp32":
                mesh.ensure_grad32()
        # the PCG reads -R from b and writes its solution straight into du
        self.b = torch.empty(n, **f64)
        # batch: a BatchExecutor that runs this workspace's PCG solves together with other threads' (the
        # handle then needs no graph of its own and takes the executor's block cap)
        self.batch = batch
        if batch is not None:
            use_graph, pcg_form, max_blocks = 0, "gather", batch.max_blocks
        self.mg = None
        if preconditioner == "multigrid":
            # geometric multigrid V-cycle (structured meshes) inside a PCG driven from the host
            from difffea_b200.multigrid import Multigrid
            self.mg = Multigrid(mesh, params)
            self.pcg = None
        else:
            self.pcg = DevicePCG(mesh, self.C, self.diag if self.blocks is None else self.blocks, self.b, self.du,
                                 use_graph=use_graph, form=pcg_form_for(mesh, pcg_form), moduli=self.moduli_kind,
                                 max_blocks=max_blocks, preconditioner=preconditioner)
        self.work = mesh.reduce_work()
        self.theta = None
        self.n_launch_groups = 0

    # ---------------------------------------------------------------------------------------------
    def set_theta(self, theta):
        _require_cuda(theta)
        if theta.numel() != self.mesh.n_el or theta.device != self.mesh.device:
            raise ValueError(f"theta must have one entry per element ({self.mesh.n_el}) on {self.mesh.device}")
        self.theta = theta.detach().to(torch.float64).contiguous()

    def residual(self, u, load_factor, out, energy=False):
        """out = R(u) (FP64); returns ||R|| (and the strain energy if asked) as Python floats."""
        _lib.call("dfea_residual_mat", self.mesh.view_ref, ptr(u), ptr(self.theta), self.material, ptr(self.f),
                  float(load_factor), ptr(out), ptr(self.scal), ptr(self.scal[1:]) if energy else ptr(None),
                  ptr(self.work), stream_handle())
        self.scal_host.copy_(self.scal, non_blocking=True)
        torch.cuda.current_stream().synchronize()
        rn = float(self.scal_host[0]) ** 0.5
        return (rn, float(self.scal_host[1])) if energy else rn

    def linearize(self, u):
        """Kernel (a): moduli C and the preconditioner at u (into the buffers the PCG graph is bound to)."""
        _lib.call("dfea_qp_moduli_mat", self.mesh.view_ref, ptr(u), ptr(self.theta), self.material, ptr(self.C),
                  self.moduli_code, ptr(self.diag), ptr(self.blocks), stream_handle())
        if self.mg is not None:
            self.mg.setup(self.C, self.moduli_code, self.diag)

    def solve(self, R, rtol, max_iter):
        """du = PCG(A, -R) to relative tolerance rtol; returns (du (FP64 buffer), iterations, status)."""
        torch.neg(R, out=self.b)
        if self.mg is not None:
            iters, status = self.mg.pcg(self.b, self.du, rtol, max_iter)
        elif self.batch is not None:
            iters, status = self.batch.solve(self.pcg, rtol, max_iter)
        else:
            iters, status = self.pcg.solve(rtol, max_iter)
        return self.du, iters, status

    def trial(self, u, alpha, du, out):
        _lib.call("dfea_add_scaled", self.mesh.n_dof, ptr(u), float(alpha), ptr(du), ptr(out), stream_handle())
        return out


def workspace_for(params, precision="fp64", cache=None):
    """A workspace for ``params`` (reused through ``cache`` if given: a dict kept by the caller)."""
    if cache is not None:
        key = (id(params["conn"]), id(params["m"]), id(params["f"]), precision)
        ws = cache.get(key)
        if ws is not None and ws.params["conn"] is params["conn"]:
            return ws
        ws = NewtonWorkspace(params, precision)
        cache[key] = ws
        return ws
    return NewtonWorkspace(params, precision)
