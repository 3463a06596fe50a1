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

from difffea_b200 import _lib, ops
from difffea_b200.cuda_mesh import _require_cuda, cuda_mesh
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
                 preconditioner="jacobi", batch=None, mg_graphs=True, mg_bounds_every=0, mg_gather=False):
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
            self.mg = Multigrid(mesh, params, graphs=mg_graphs, bounds_every=mg_bounds_every, gather=mg_gather)
            self.pcg = None
        else:
            self.pcg = DevicePCG(mesh, self.C, self.diag if self.blocks is None else self.blocks, self.b, self.du,
                                 use_graph=use_graph, form=pcg_form_for(mesh, pcg_form), moduli=self.moduli_kind,
                                 max_blocks=max_blocks, preconditioner=preconditioner)
        self.work = mesh.reduce_work()
        self.mesh_id = ops.register_mesh(mesh)
        self.mat_args = ops.material_args(self.material)
        self._empty = torch.empty(0, dtype=torch.float64, device=dev)
        self.id = ops.register_handle(self)
        self.theta = None
        self.n_launch_groups = 0
        self._native = None           # the dfea_newton description, built on the first native solve

    # ---------------------------------------------------------------------------------------------
    def retarget(self, params):
        """
        Bind this workspace to another problem on the same mesh (the same conn, geometry and supports): its
        load vector and material replace the current ones; every device buffer, the bound PCG graph and the
        multigrid hierarchy are kept.
        """
        for k in ("conn", "dN_dX", "w_detJ", "m"):
            if params[k] is not self.params[k]:
                raise ValueError(f"retarget needs the same mesh: params['{k}'] differs")
        self.params = params
        self.f.copy_(params["f"].detach().to(torch.float64))
        self.material = device_material(params)
        self.mat_args = ops.material_args(self.material)

    def set_theta(self, theta):
        _require_cuda(theta)
        if theta.numel() != self.mesh.n_el or theta.device != self.mesh.device:
            raise ValueError(f"theta must have one entry per element ({self.mesh.n_el}) on {self.mesh.device}")
        self.theta = theta.detach().to(torch.float64).contiguous()

    def residual(self, u, load_factor, out, energy=False):
        """out = R(u) (FP64); returns ||R|| (and the strain energy if asked) as Python floats."""
        torch.ops.difffea_b200.residual_out(self.mesh_id, u, self.theta, *self.mat_args, self.f, float(load_factor),
                                            out, self.scal, bool(energy))
        self.scal_host.copy_(self.scal, non_blocking=True)
        torch.cuda.current_stream().synchronize()
        rn = float(self.scal_host[0]) ** 0.5
        return (rn, float(self.scal_host[1])) if energy else rn

    def linearize(self, u):
        """Kernel (a): moduli C and the preconditioner at u (into the buffers the PCG graph is bound to)."""
        torch.ops.difffea_b200.qp_moduli_out(self.mesh_id, u, self.theta, *self.mat_args, self.C, self.moduli_code,
                                             self.diag, self.blocks if self.blocks is not None else self._empty)
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

    # ---------------------------------------------------------------------------------------------
    # the whole solve in the library's C++ driver (dfea_newton_solve, custom op newton_solve)
    # ---------------------------------------------------------------------------------------------
    MAX_RECORDS = 1024

    def native_solve(self, theta, n_load_steps, tol, max_newton=25, max_cutbacks=8, pcg_max_iter=500):
        """
        newton_krylov_solve's loop in C++ on this workspace's buffers (one call, no interpreter lock held):
        returns (u (2N,) float64, info) with the reference's info keys; ``history`` holds the Newton records
        (at most MAX_RECORDS), ``snapshots`` the initial and the final state only.
        """
        if self.batch is not None:
            raise ValueError("the native driver runs its own PCG; a workspace bound to a BatchExecutor cannot use it")
        self.set_theta(theta)
        if self._native is None:
            self._build_native()
        u, stats = torch.ops.difffea_b200.newton_solve(self.id, self.theta, int(n_load_steps), float(tol),
                                                        int(max_newton), int(max_cutbacks), int(pcg_max_iter))
        converged, load_factor, total_newton, total_cg, n_cutbacks, n_records = stats.tolist()
        history = [dict(step=r.step, load_factor=r.load_factor, iteration=r.iteration, residual=r.residual,
                        cg_iters=r.cg_iters, alpha=r.alpha) for r in self._records[:int(n_records)]]
        return u, {"converged": bool(converged), "load_factor": float(load_factor), "history": history,
                   "total_newton": int(total_newton), "total_cg": int(total_cg), "n_cutbacks": int(n_cutbacks),
                   "snapshots": [(0.0, torch.zeros_like(u)), (float(load_factor), u.clone())]}

    def _build_native(self):
        import ctypes
        mesh, n, dev = self.mesh, self.mesh.n_dof, self.mesh.device
        f64 = dict(dtype=torch.float64, device=dev)
        self.w = torch.empty(n, **f64)
        uD = self.params.get("u_D")
        self.u_D = None if uD is None or not bool((uD != 0).any()) else uD.detach().to(**f64).contiguous()
        self._records = (_lib.NewtonRecord * self.MAX_RECORDS)()
        nw = _lib.Newton()
        nw.mesh = ctypes.pointer(mesh.view)
        for name, t in (("f", self.f), ("u_D", self.u_D), ("w", self.w), ("uc", self.uc), ("R", self.R),
                        ("Rc", self.Rc), ("du", self.du), ("b", self.b), ("diag", self.diag), ("blocks", self.blocks),
                        ("moduli", self.C), ("reduce_work", self.work), ("scal", self.scal),
                        ("scal_host", self.scal_host)):
            setattr(nw, name, t.data_ptr() if t is not None else None)
        nw.moduli_dtype = self.moduli_code
        if self.mg is not None:
            nw.mg = ctypes.pointer(self.mg.h)
        else:
            nw.pcg = self.pcg._h.value
        from difffea_b200.newton_krylov import FP32_MIN_RTOL
        nw.min_rtol = FP32_MIN_RTOL if self.precision == "fp32" else 0.0
        self._native = nw

    def _native_args(self, theta):
        """The dfea_newton description for a solve at theta (this workspace's buffers) and a fresh u."""
        self.set_theta(theta)
        if self._native is None:
            self._build_native()
        nw = self._native
        nw.material = self.material
        nw.theta = self.theta.data_ptr()
        u = torch.empty(self.mesh.n_dof, dtype=torch.float64, device=self.mesh.device)
        nw.u = u.data_ptr()
        return nw, u

    def trial(self, u, alpha, du, out):
        torch.ops.difffea_b200.add_scaled_out(u, float(alpha), du, out)
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
