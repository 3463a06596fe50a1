"""
Per-kernel microbenchmarks on structured rectangle meshes (CUDA-event timed, L2 flushed between
launches unless ``--no-flush``).

    python -m difffea_b200.microbench sweep                       tangent product: Q4/Q9 x 40k..2.56M x fp64/fp32
    python -m difffea_b200.microbench apply --element quad4 --elements 640000 --precision fp64
    python -m difffea_b200.microbench moduli|residual|sensitivity|fields|pcg --element quad4 --elements 640000
                                            [--material mooney_rivlin|...|all]
    python -m difffea_b200.microbench vcycle --element quad4 --elements 1048576
                                            multigrid set-up and one V-cycle (structured mesh)
    python -m difffea_b200.microbench solve --element quad4 --nx 256 --precision mixed
                                            one serving request (4:1 cantilever, E 1, nu 0.3, load 0.03)
                                            solved twice; the second solve is timed
    --form gather                           the gather form of the product (element pass + node sums)
                                            for apply, pcg, solve and sweep

State: nodal displacements uniform in +-0.05 h on free DOFs (seeded), input vector N(0, 1), E = 1,
nu = 0.3, h = 1.  Algorithmic bytes count every array a kernel must touch once:

    apply        moduli n_el n_q 16 s_C + gradients n_el n_q nen 2 s_G + connectivity n_el nen 4
                 + vectors 3 x 2N s_v (v read, y initialised, y written)
    moduli       connectivity + gradients (FP64) + w detJ n_el n_q 8 + theta n_el 8 + u 2N 8
                 + moduli written n_el n_q 16 s_C + diagonal 2 x 2N 8
    residual     connectivity + gradients + w detJ + theta + u, f read + R written (3 x 2N 8)
    sensitivity  connectivity + gradients + w detJ + u, lambda read (2 x 2N 8) + g written n_el 8
    fields       connectivity + gradients + w detJ + theta + u + 7 element rows written (n_el 56)
    pcg          per iteration: the product with the curvature fused (apply bytes) + update 1 (7 vectors)
                 + update 2 (5 vectors + N fix bytes)

``precision``: fp64 (FP64 moduli, gradients and vectors), fp32 (all FP32), mixed (FP32 moduli and
gradients on FP64 vectors) or ref (FP32 moduli in the element reference frame, 10 per Gauss point, on
FP64 vectors: the serving operator; the product reads no gradients, its bytes count 10 moduli).
"""
import argparse
import json
import os

import torch

from difffea_b200 import _lib, ops
from difffea_b200.cuda_mesh import cuda_mesh, ptr, stream_handle
from difffea_b200.materials import MATERIAL_LIBRARY, device_material
from difffea_b200.problem import build_rectangle_problem

NEN = {"quad4": 4, "quad9": 9}
NQ = {"quad4": 4, "quad9": 9}
SWEEP_ELEMENTS = (40_000, 160_000, 640_000, 2_560_000)
_SIZES = {"fp64": (8, 8, 8), "fp32": (4, 4, 4), "mixed": (4, 4, 8), "ref": (4, 0, 8)}  # (moduli, gradients, vectors)


def side_for(n_elements):
    n = int(round(n_elements ** 0.5))
    if n * n != n_elements:
        raise ValueError("the structured meshes here are square: n_elements must be a perfect square")
    return n


class State:
    """A square n x n mesh of unit cells with a seeded state, its packed mesh and moduli."""

    def __init__(self, element, n_elements, precision="fp64", device="cuda", seed=0, form="colour",
                 material="neo_hookean"):
        n = side_for(n_elements)
        self.form = form
        self.element, self.precision, self.device = element, precision, torch.device(device)
        self.p = build_rectangle_problem(element, n, n, float(n), float(n), E=1.0, nu=0.3, device=device,
                                         build_on_device=True, material=material)
        g = torch.Generator().manual_seed(seed)
        N2 = self.p["f"].shape[0]
        self.N2 = N2
        self.u = (((torch.rand(N2, dtype=torch.float64, generator=g) * 2 - 1) * 0.05).to(device)) * self.p["m"]
        self.theta = torch.ones(self.p["conn"].shape[0], dtype=torch.float64, device=device)
        self.mesh = cuda_mesh(self.p)
        self.mid = ops.register_mesh(self.mesh)
        self.mat = device_material(self.p)
        fp32_C = precision in ("fp32", "mixed")
        if fp32_C:
            self.mesh.ensure_grad32()
        if precision == "ref":
            self.mesh.ensure_ref_frame()
            self.C = torch.empty(self.mesh.moduli_numel_ref(), dtype=torch.float32, device=device)
            self.diag = torch.empty(N2, dtype=torch.float64, device=device)
            _lib.call("dfea_qp_moduli_mat", self.mesh.view_ref, ptr(self.u), ptr(self.theta), self.mat,
                      ptr(self.C), _lib.DFEA_F32REF, ptr(self.diag), ptr(None), stream_handle())
        else:
            self.C, self.diag = ops.qp_moduli(self.mid, self.u, self.theta, *ops.material_args(self.mat), fp32_C,
                                              True)
        vt = torch.float32 if precision == "fp32" else torch.float64
        pad = (N2 + 63) // 64 * 64
        self.buf = torch.empty(2 * pad, dtype=vt, device=device)            # [v | y], as the PCG's vectors
        self.v, self.y = self.buf[:N2], self.buf[pad:pad + N2]
        self.v.copy_(torch.randn(N2, dtype=torch.float64, generator=g).to(device))
        self.n_el = self.p["conn"].shape[0]
        self.nen, self.nq = self.p["conn"].shape[1], self.p["dN_dX"].shape[1]
        self.fe = None
        if form in ("gather", "fused"):
            self.mesh.ensure_node_incidence()
            vcode = _lib.DFEA_F32 if vt == torch.float32 else _lib.DFEA_F64
            nbytes = int(_lib.load().dfea_gather_work_bytes(self.mesh.view_ref, vcode))
            self.fe = torch.empty(nbytes, dtype=torch.uint8, device=device)

    # algorithmic bytes ----------------------------------------------------------------------------
    def apply_bytes(self):
        """Bytes the product must move; the gather form is charged the colour form's minimum (its element
        results and incidence are extra traffic it pays for fewer launches)."""
        sC, sG, sv = _SIZES[self.precision]
        n_c = 10 if self.precision == "ref" else 16
        return (self.n_el * self.nq * n_c * sC + self.n_el * self.nq * self.nen * 2 * sG
                + self.n_el * self.nen * 4 + 3 * self.N2 * sv)

    def _geometry_bytes(self):
        return self.n_el * self.nen * 4 + self.n_el * self.nq * self.nen * 2 * 8 + self.n_el * self.nq * 8

    def moduli_bytes(self):
        sC = _SIZES[self.precision][0]
        return (self._geometry_bytes() + self.n_el * 8 + self.N2 * 8 + self.n_el * self.nq * 16 * sC
                + 2 * self.N2 * 8)

    def residual_bytes(self):
        return self._geometry_bytes() + self.n_el * 8 + 3 * self.N2 * 8

    def sensitivity_bytes(self):
        return self._geometry_bytes() + 2 * self.N2 * 8 + self.n_el * 8

    def fields_bytes(self):
        return self._geometry_bytes() + self.n_el * 8 + self.N2 * 8 + 7 * self.n_el * 8

    def pcg_bytes_per_iteration(self):
        sv = _SIZES[self.precision][2]
        return self.apply_bytes() + 12 * self.N2 * sv + self.N2 // 2

    # launches ---------------------------------------------------------------------------------------
    def apply(self):
        cdt = _lib.DFEA_F64 if self.C.dtype == torch.float64 else _lib.DFEA_F32
        if self.precision == "ref":
            cdt = _lib.DFEA_F32REF
        vdt = _lib.DFEA_F64 if self.v.dtype == torch.float64 else _lib.DFEA_F32
        if self.form in ("gather", "fused"):
            _lib.call("dfea_tangent_apply_gather", self.mesh.view_ref, ptr(self.C), cdt, ptr(self.v), ptr(self.y), vdt,
                      ptr(self.fe), stream_handle())
        else:
            _lib.call("dfea_tangent_apply", self.mesh.view_ref, ptr(self.C), cdt, ptr(self.v), ptr(self.y), vdt,
                      stream_handle())

    def moduli(self):
        if self.precision == "ref":
            _lib.call("dfea_qp_moduli_mat", self.mesh.view_ref, ptr(self.u), ptr(self.theta), self.mat,
                      ptr(self.C), _lib.DFEA_F32REF, ptr(self.diag), ptr(None), stream_handle())
        else:
            ops.qp_moduli(self.mid, self.u, self.theta, *ops.material_args(self.mat), self.precision != "fp64", True)

    def residual(self):
        ops.residual(self.mid, self.u, self.theta, *ops.material_args(self.mat), self.p["f"], 1.0)

    def sensitivity(self):
        ops.element_sensitivity(self.mid, self.u, self.v.double(), *ops.material_args(self.mat))

    def fields(self):
        if getattr(self, "el_fields", None) is None:
            self.el_fields = torch.empty(7, self.n_el, dtype=torch.float64, device=self.device)
        _lib.call("dfea_element_fields_mat", self.mesh.view_ref, ptr(self.u), ptr(self.theta), self.mat,
                  ptr(self.el_fields), stream_handle())


def time_launches(fn, reps=20, warmup=3, flush=True, device="cuda"):
    """Mean and min milliseconds of ``fn`` (CUDA events on the launching stream, one pair per launch)."""
    scratch = torch.empty(256 * 2 ** 20, dtype=torch.uint8, device=device) if flush else None
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    s = torch.cuda.current_stream()
    times = []
    for _ in range(reps):
        if scratch is not None:
            scratch.fill_(1)                                   # 256 MB > L2: evict the previous launch's lines
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        fn()
        e1.record(s)
        times.append((e0, e1))
    torch.cuda.synchronize()
    ms = [a.elapsed_time(b) for a, b in times]
    return sum(ms) / len(ms), min(ms)


def hbm_peak():
    here = os.path.dirname(os.path.abspath(__file__))
    for path in (os.path.join(here, "..", "..", "MEASURED_PEAKS.json"), "MEASURED_PEAKS.json"):
        if os.path.exists(path):
            with open(path) as fh:
                return float(json.load(fh)["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def measure(kind, element, n_elements, precision, reps=20, flush=True, pcg_iters=64, pcg_graph=1, form="colour",
            material="neo_hookean"):
    st = State(element, n_elements, precision, form=form, material=material)
    peak, peak_kind = hbm_peak()
    row = dict(kernel=kind, element=element, n_el=st.n_el, precision=precision, colours=st.mesh.n_colours, form=form,
               material=material)
    if kind == "pcg":
        from difffea_b200.krylov import DevicePCG
        vt = st.v.dtype
        d = st.diag.to(vt)
        b = (st.p["m"].to(vt) * st.v).contiguous()
        x = torch.empty_like(b)
        solver = DevicePCG(st.mesh, st.C, d, b, x, use_graph=pcg_graph, form=form,
                           moduli="ref" if precision == "ref" else "physical")

        def fn():
            solver.solve(1e-30, pcg_iters)                     # exactly pcg_iters iterations
        ms, ms_min = time_launches(fn, reps=max(3, reps // 4), flush=flush)
        solver.close()
        nbytes = st.pcg_bytes_per_iteration()
        row.update(pcg_graph=solver.use_graph, ms_per_iteration=ms / pcg_iters, bytes_per_iteration=nbytes,
                   gbs=nbytes / (ms / pcg_iters * 1e-3) / 1e9)
    else:
        fn = getattr(st, kind)
        nbytes = getattr(st, f"{kind}_bytes")()
        ms, ms_min = time_launches(fn, reps=reps, flush=flush)
        row.update(ms=ms, ms_min=ms_min, bytes=nbytes, gbs=nbytes / (ms * 1e-3) / 1e9)
    row.update(frac=row["gbs"] / peak, peak_gbs=peak, peak_kind=peak_kind)
    del st
    torch.cuda.empty_cache()
    return row


def vcycle_once(element, n_elements, precision, reps=10, gather=False):
    """Set-up and one V-cycle of the multigrid preconditioner on the microbench mesh (CUDA events); ``gather``:
    level 0 in the gather form (the serving engine's)."""
    from difffea_b200.multigrid import Multigrid
    st = State(element, n_elements, precision)
    code = _lib.DFEA_F32REF if precision == "ref" else (_lib.DFEA_F64 if st.C.dtype == torch.float64 else _lib.DFEA_F32)
    mg = Multigrid(st.mesh, st.p, gather=gather)
    r = torch.randn(st.N2, dtype=torch.float64, generator=torch.Generator().manual_seed(1)).to(st.device)
    z = torch.empty_like(r)
    setup_ms, _ = time_launches(lambda: mg.setup(st.C, code, st.diag), reps=3, warmup=1)
    cycle_ms, cycle_min = time_launches(lambda: mg.apply(r, z), reps=reps)
    return dict(kernel="vcycle", element=element, n_el=st.n_el, precision=precision,
                levels=[(lv.gx, lv.gy) for lv in mg.levels], setup_ms=setup_ms, cycle_ms=cycle_ms, cycle_ms_min=cycle_min)


def solve_once(element, nx, precision, pcg_graph, form="auto", preconditioner="jacobi", mg_graphs=False,
               mg_bounds_every=3, mg_gather=False):
    """Wall and device milliseconds of one serving-type request (the second of two identical solves)."""
    import time
    from difffea_b200.serving import Request, solve_request
    req = Request(0, element, nx, 1.0, 0.3, 0.03)
    prec = "fp64" if precision == "fp64" else "fp32"     # the solver's "fp32" is the mixed operator
    out = {}
    for k in range(2):
        s = torch.cuda.current_stream()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        t = time.perf_counter()
        e0.record(s)
        u, info = solve_request(req, "cuda", precision=prec, pcg_graph=pcg_graph, pcg_form=form,
                                preconditioner=preconditioner, mg_graphs=mg_graphs, mg_bounds_every=mg_bounds_every,
                                mg_gather=mg_gather)
        e1.record(s)
        torch.cuda.synchronize()
        out = dict(kernel="solve", element=element, nx=nx, n_el=req.n_elements, precision=precision,
                   pcg_graph=pcg_graph, form=form, preconditioner=preconditioner, newton=info["total_newton"],
                   cg=info["total_cg"],
                   converged=info["converged"], device_ms=e0.elapsed_time(e1),
                   wall_ms=1e3 * (time.perf_counter() - t))
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m difffea_b200.microbench")
    ap.add_argument("kind", choices=("sweep", "apply", "moduli", "residual", "sensitivity", "fields", "pcg", "solve",
                                     "vcycle"))
    ap.add_argument("--element", default="quad4", choices=tuple(NEN))
    ap.add_argument("--elements", type=int, default=640_000)
    ap.add_argument("--precision", default="fp64", choices=tuple(_SIZES))
    ap.add_argument("--reps", type=int, default=20)
    ap.add_argument("--pcg-iters", type=int, default=64)
    ap.add_argument("--no-flush", action="store_true")
    ap.add_argument("--nx", type=int, default=256)
    ap.add_argument("--sweep-precisions", default="fp64,fp32", help="comma-separated precisions of the sweep")
    ap.add_argument("--form", default=None, choices=("colour", "gather", "fused", "auto"),
                    help="product form: one launch per colour, or element pass + node sums (default: colour; "
                         "for solve, auto = the solver's choice by mesh size)")
    ap.add_argument("--material", default="neo_hookean", choices=tuple(MATERIAL_LIBRARY) + ("all",),
                    help="material of the moduli / residual / sensitivity / fields kernels (library defaults); "
                         "all = every material in turn")
    ap.add_argument("--preconditioner", default="jacobi", choices=("jacobi", "block_jacobi", "multigrid"),
                    help="preconditioner of the solve kind")
    ap.add_argument("--mg-graphs", action="store_true", help="solve: graph-driven multigrid (default: host-driven, "
                    "as the serving engine)")
    ap.add_argument("--mg-bounds-every", type=int, default=3, help="solve: multigrid smoother bounds every k-th set-up")
    ap.add_argument("--mg-gather", action="store_true", help="vcycle / solve: level 0 of the hierarchy in the gather form")
    ap.add_argument("--pcg-graph", type=int, default=None,
                    help="PCG form: 0 direct launches (solve's default), 1 loop graph (pcg's default), "
                         "2 unrolled graph")
    a = ap.parse_args(argv)
    if a.kind == "solve":
        print(json.dumps(solve_once(a.element, a.nx, a.precision, 0 if a.pcg_graph is None else a.pcg_graph,
                                    a.form or "auto", a.preconditioner, a.mg_graphs, a.mg_bounds_every, a.mg_gather)),
              flush=True)
        return 0
    if a.kind == "vcycle":
        print(json.dumps(vcycle_once(a.element, a.elements, a.precision, a.reps, gather=a.mg_gather)), flush=True)
        return 0
    if a.kind == "sweep":
        for element in ("quad4", "quad9"):
            for prec in a.sweep_precisions.split(","):
                for n in SWEEP_ELEMENTS:
                    print(json.dumps(measure("apply", element, n, prec, a.reps, not a.no_flush, form=a.form or "colour")),
                          flush=True)
        return 0
    for material in (MATERIAL_LIBRARY if a.material == "all" else (a.material,)):
        print(json.dumps(measure(a.kind, a.element, a.elements, a.precision, a.reps, not a.no_flush, a.pcg_iters,
                                 1 if a.pcg_graph is None else a.pcg_graph, a.form or "colour", material)),
              flush=True)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
