"""
Continuous-batching serving of Newton-Krylov solves on one GPU.

A request is a structured 4:1 cantilever bar (Q4 or Q9, nx x nx/4 cells on [0, 4] x [0, 1]), clamped at
x = 0 and pulled at x = 4 by a uniform dead traction of `load` per unit length (axial stress ~ load, strain
~ load / E), neo-Hookean with (E, nu).  ``request_stream`` draws the seeded stream: nx uniform over the
multiples of 4 in [16, 512], Q4/Q9 with equal probability, E log-uniform in [0.5, 2], nu uniform in
[0.2, 0.45], load uniform in [0.01, 0.05], Poisson arrivals.

``ServingEngine`` runs requests in *slots*.  Every slot is a worker with its own CUDA stream; an admitted
request is built on the device, solved by the device-resident Newton-Krylov solver (FP32 moduli and PCG
inside an FP64 Newton loop by default: residual, line search, convergence test and state update in
FP64), and its displacement copied back.  Each PCG solve is one CUDA graph with a device-side loop, so a
slot needs the host only between Newton steps, and the kernels of all slots overlap on the GPU: a
request that arrives while others run starts as soon as a slot and enough HBM are free (admission by
an HBM budget), its work interleaving with theirs.  Solves are deterministic and independent, so a
request's result does not depend on what else is in flight.
"""
import math
import queue
import threading
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from difffea_b200.newton_krylov import newton_krylov_solve
from difffea_b200.problem import build_rectangle_problem
from difffea_b200.workspace import NewtonWorkspace

NEN = {"quad4": 4, "quad9": 9}
NQ = {"quad4": 4, "quad9": 9}


@dataclass
class Request:
    rid: int
    element_type: str
    nx: int
    E: float
    nu: float
    load: float
    arrival: float = 0.0          # seconds after the stream starts

    @property
    def ny(self):
        return self.nx // 4

    @property
    def n_elements(self):
        return self.nx * self.ny

    @property
    def n_nodes(self):
        k = 2 if self.element_type == "quad9" else 1
        return (k * self.nx + 1) * (k * self.ny + 1)

    def validate(self):
        """Raise ValueError for a request the solver cannot take (checked on the host before any GPU work)."""
        if self.element_type not in NEN:
            raise ValueError(f"request {self.rid}: element type '{self.element_type}' is not served ({sorted(NEN)})")
        if not (isinstance(self.nx, int) and self.nx >= 4 and self.nx % 4 == 0):
            raise ValueError(f"request {self.rid}: nx must be a positive multiple of 4, got {self.nx}")
        if not (math.isfinite(self.E) and self.E > 0):
            raise ValueError(f"request {self.rid}: E must be finite and positive, got {self.E}")
        if not (math.isfinite(self.nu) and 0.0 <= self.nu < 0.5):
            raise ValueError(f"request {self.rid}: nu must lie in [0, 0.5), got {self.nu}")
        if not math.isfinite(self.load):
            raise ValueError(f"request {self.rid}: load must be finite, got {self.load}")


@dataclass
class Result:
    rid: int
    u: torch.Tensor = None        # host (2N,) float64
    converged: bool = False
    newton: int = 0
    cg: int = 0
    admitted: float = 0.0
    finished: float = 0.0
    arrival: float = 0.0
    error: str = ""
    load_factor: float = 0.0      # the load factor reached (1.0 when converged)
    extra: dict = field(default_factory=dict)

    @property
    def latency(self):
        return self.finished - self.arrival


def request_stream(n=2000, seed=0, rate=None):
    """The seeded request stream; arrivals are Poisson with ``rate`` requests/s (all at t = 0 if None)."""
    rng = np.random.default_rng(seed)
    nxs = rng.choice(np.arange(16, 513, 4), size=n)
    types = np.where(rng.random(n) < 0.5, "quad4", "quad9")
    Es = np.exp(rng.uniform(np.log(0.5), np.log(2.0), size=n))
    nus = rng.uniform(0.2, 0.45, size=n)
    loads = rng.uniform(0.01, 0.05, size=n)
    gaps = rng.exponential(1.0, size=n)
    out = []
    t = 0.0
    for i in range(n):
        if rate is not None:
            t += gaps[i] / rate
        out.append(Request(i, str(types[i]), int(nxs[i]), float(Es[i]), float(nus[i]), float(loads[i]),
                           arrival=t if rate is not None else 0.0))
    return out


def with_arrivals(requests, rate, seed=1):
    """Copies of ``requests`` with Poisson arrival times at ``rate`` requests/s."""
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    for r in requests:
        t += rng.exponential(1.0 / rate)
        out.append(Request(r.rid, r.element_type, r.nx, r.E, r.nu, r.load, arrival=t))
    return out


# "auto" preconditioner: geometric multigrid from this many nodes up (structured rectangles), Jacobi below.
# Measured crossover on B200 (one request, FP32 operator, 1 load step, tol 1e-10 ||f||): Q4 64 x 16 (1,105
# nodes) 15.6 ms Jacobi vs 18.1 ms multigrid, Q4 128 x 32 (4,257) 28.2 vs 21.0, Q9 64 x 16 (4,257) 40.0 vs
# 24.0, Q9 512 x 128 (263,169) 381 vs 49.
MULTIGRID_MIN_NODES = 2500


def preconditioner_for(req, preconditioner="auto"):
    """The preconditioner a request is solved with: "auto" picks multigrid for the larger requests."""
    if preconditioner != "auto":
        return preconditioner
    return "multigrid" if req.n_nodes >= MULTIGRID_MIN_NODES else "jacobi"


def hbm_estimate(req, precision="fp32", preconditioner="jacobi"):
    """Bytes a request holds on the device while it runs (problem, packed mesh, moduli, vectors)."""
    E, N = req.n_elements, req.n_nodes
    nen, nq = NEN[req.element_type], NQ[req.element_type]
    per_el = (8 * nen + 16 * nq * nen + 8 * nq          # problem dictionary: conn, dN_dX, w_detJ
              + 4 * nen + 4 + 16 * nq * nen + 8 * nq + 8  # packed mesh (FP64 gradients)
              + ((40 + 32) * nq if precision == "fp32"  # reference-frame FP32 moduli + inverse Jacobians
                 else 128 * nq)                         # FP64 moduli
              + 16 * nen + 4 * nen                      # gather form: element results, node incidence
              + 32 * nen)                               # int64 keys, values and order of the incidence sort
    per_node = 16 + 2 * 8 * 14 + 2 * 4 * 6 + 1 + 4      # nodes, ~14 f64 and ~6 f32 DOF vectors, fix bits, ptr
    if preconditioner_for(req, preconditioner) == "multigrid":
        # 10 FP64 DOF vectors on the fine grid (6 of the cycle, 4 of its PCG), a third more over the coarse
        # levels, their 8 x 8 element matrices (a quarter of the fine cells at level 1, Q9: as many), grid maps
        cells1 = E if NEN[req.element_type] == 9 else E / 4
        per_node += 10 * 16 * 4 / 3 + 8 + 4
        # the grid inference's int64 temporaries (connectivity built per candidate numbering, grid maps)
        per_el += 8 * nen + 96
        per_node += 96
        return int(1.1 * (E * per_el + N * per_node + cells1 * 512 * 4 / 3) + 4 * 2 ** 20)
    return int(E * per_el + N * per_node + 4 * 2 ** 20)  # + reduction scratch and PCG state


def pcg_iteration_bytes(req):
    """
    Bytes one PCG iteration of a request must move in the serving configuration (reference-frame FP32
    moduli, gather form, FP64 Krylov vectors): per element the moduli (40 B per Gauss point) and the
    connectivity, the element results written and read back (2 x 16 B per local node) and the incidence
    (4 B per local node); per node 11 passes over FP64 pairs (the gather of p, update 1 reading p, d, x,
    r and writing x, r, update 2 reading r, d, p and writing p), the incidence pointer and the fix byte.
    """
    nen, nq = NEN[req.element_type], NQ[req.element_type]
    per_el = 40 * nq + 4 * nen + 32 * nen + 4 * nen
    per_node = 11 * 16 + 4 + 1
    return req.n_elements * per_el + req.n_nodes * per_node


def request_problem(req, device="cpu", build_on_device=False, pin_memory=False):
    """
    The problem dictionary of a request (on ``device``).  A Q4 or Q9 request's arrays are written by one library
    call -- on the GPU (``dfea_build_rectangle``, with ``build_on_device``) or on the host
    (``dfea_build_rectangle_host``, ``device="cpu"``; into page-locked memory with ``pin_memory``, ready to be
    copied): the mesh, supports and load of build_rectangle_problem, its geometry and load vector to rounding
    (the sums run in another order), with no torch operations -- the serving engine's slots then hold the
    interpreter lock for less of each request.
    """
    dev = torch.device(device)
    if req.element_type in _RECT_NEN:
        if dev.type == "cuda" and build_on_device:
            return _device_request_problem(req, dev)
        if dev.type == "cpu":
            return _host_request_problem(req, pin_memory)
    p = build_rectangle_problem(req.element_type, req.nx, req.ny, 4.0, 1.0, E=req.E, nu=req.nu,
                                load=(req.load * 1.0, 0.0), device=device, build_on_device=build_on_device)
    return {k: (v.pin_memory() if torch.is_tensor(v) else v) for k, v in p.items()} if pin_memory else p


def reference_request_problem(req):
    """The problem dictionary of a request built on the host by build_rectangle_problem (torch operations, the
    reference's problem construction restated), independently of the library's builders: the input of the
    reference arm and of the parity checks."""
    return build_rectangle_problem(req.element_type, req.nx, req.ny, 4.0, 1.0, E=req.E, nu=req.nu,
                                   load=(req.load * 1.0, 0.0))


_RECT_NEN = {"quad4": 4, "quad9": 9}
_RECT_TEMPLATES = {}


def _rect_template(element_type):
    """The element type's quadrature data in a ``dfea_rect_spec`` (built once per element type)."""
    spec = _RECT_TEMPLATES.get(element_type)
    if spec is None:
        from difffea_b200 import _lib
        from difffea_b200.elements import element_quadrature, gauss_1d, quadrature_gradients
        GP, GW = element_quadrature(element_type)
        s, w = gauss_1d(3)
        spec = _lib.RectSpec()
        spec.nen, spec.n_q = _RECT_NEN[element_type], GW.numel()
        for i, x in enumerate(quadrature_gradients(element_type, GP).reshape(-1).tolist()):
            spec.ref_grad[i] = x
        for i, x in enumerate(GW.tolist()):
            spec.gauss_w[i] = x
        for i in range(3):
            spec.edge_s[i], spec.edge_w[i] = float(s[i]), float(w[i])
        spec = _RECT_TEMPLATES.setdefault(element_type, spec)
    return spec


def _rect_arrays(req, **kw):
    """A request's dfea_rect_spec and empty arrays for the builder (torch.empty keywords ``kw``)."""
    from difffea_b200 import _lib
    spec = _lib.RectSpec.from_buffer_copy(_rect_template(req.element_type))
    spec.nx, spec.ny, spec.width, spec.height = req.nx, req.ny, 4.0, 1.0
    spec.load_x, spec.load_y = req.load * 1.0, 0.0
    nen, nq, span = spec.nen, spec.n_q, (2 if spec.nen == 9 else 1)
    N, n_el = (span * req.nx + 1) * (span * req.ny + 1), req.nx * req.ny
    f64 = dict(dtype=torch.float64, **kw)
    arrays = dict(nodes=torch.empty(N, 2, **f64), conn=torch.empty(n_el, nen, dtype=torch.int64, **kw),
                  dN_dX=torch.empty(n_el, nq, nen, 2, **f64), w_detJ=torch.empty(n_el, nq, **f64),
                  f=torch.empty(2 * N, **f64), m=torch.empty(2 * N, **f64),
                  fixed=torch.empty(2 * N, dtype=torch.bool, **kw), u_D=torch.empty(2 * N, **f64))
    return spec, arrays


def _rect_problem(req, a, GP, GW, mat_device=None):
    """The problem dictionary (build_rectangle_problem's keys, in its order) of the builder's arrays ``a``."""
    from difffea_b200.elements import make_shape_fn
    from difffea_b200.materials import lame_parameters, material_vector
    mu0, lmbda0 = lame_parameters(req.E, req.nu)
    mat_p, mat_scalable = material_vector("neo_hookean", {"mu": mu0, "lmbda": lmbda0})
    if mat_device is not None:
        mat_p, mat_scalable = mat_p.to(mat_device), mat_scalable.to(mat_device)
    return {"nodes": a["nodes"], "conn": a["conn"], "shape_fn": make_shape_fn(req.element_type), "GP": GP, "GW": GW,
            "material": "neo_hookean", "mat_p": mat_p, "mat_scalable": mat_scalable, "f": a["f"], "m": a["m"],
            "fixed": a["fixed"], "u_D": a["u_D"], "element_type": req.element_type, "dN_dX": a["dN_dX"],
            "w_detJ": a["w_detJ"]}


def _host_request_problem(req, pin_memory=False):
    import ctypes
    from difffea_b200 import _lib
    from difffea_b200.cuda_mesh import ptr
    from difffea_b200.elements import element_quadrature
    spec, a = _rect_arrays(req, pin_memory=True) if pin_memory else _rect_arrays(req)
    _lib.call("dfea_build_rectangle_host", ctypes.byref(spec), *(ptr(a[k]) for k in _RECT_ARGS))
    GP, GW = element_quadrature(req.element_type)
    return _rect_problem(req, a, GP, GW)


_RECT_ARGS = ("nodes", "conn", "dN_dX", "w_detJ", "f", "m", "fixed", "u_D")


def _device_request_problem(req, device):
    import ctypes
    from difffea_b200 import _lib
    from difffea_b200.cuda_mesh import ptr, stream_handle
    from difffea_b200.elements import element_quadrature
    if device.index is None:
        device = torch.device("cuda", torch.cuda.current_device())
    spec, a = _rect_arrays(req, device=device)
    with torch.cuda.device(device):
        _lib.call("dfea_build_rectangle", ctypes.byref(spec), *(ptr(a[k]) for k in _RECT_ARGS), stream_handle())
    GP, GW = element_quadrature(req.element_type, torch.float64, device)
    return _rect_problem(req, a, GP, GW, mat_device=device)


class PooledSolve:
    """
    A served mesh kept for the next request on it: the device problem dictionary and the solver workspace
    (packed mesh, moduli, Krylov vectors, the bound PCG graph or multigrid hierarchy and its captured graphs),
    plus what rebuilding the load vector needs.  A request on the same mesh differs only in its load
    magnitude and material, which ``retarget`` sets; the load vector comes from the same function as in a
    fresh build, so a pooled solve gives the fresh solve's result bit for bit.
    """

    def __init__(self, req, params, ws, nbytes):
        from difffea_b200.boundary_conditions import boundary_edges, select_boundary_nodes
        from difffea_b200.elements import get_element
        el = get_element(req.element_type)
        self.params, self.ws, self.nbytes = params, ws, nbytes
        self.order = el["order"]
        self.edges = boundary_edges(params["conn"], el["edges"])
        self.load_nodes = select_boundary_nodes(params["nodes"], "right")
        self.native = req.element_type in _RECT_NEN and params["nodes"].is_cuda

    def retarget(self, req):
        """The problem dictionary of ``req`` on this mesh (new load vector and material), bound to the workspace."""
        from difffea_b200.boundary_conditions import edge_traction_load
        from difffea_b200.materials import lame_parameters, material_vector
        p = self.params
        if self.native:       # the load vector the fresh build of this request would have
            f = request_problem(req, p["nodes"].device, build_on_device=True)["f"].reshape(-1, 2)
        else:
            f = edge_traction_load(p["nodes"], self.edges, self.order, self.load_nodes, (float(req.load * 1.0), 0.0))
        mu0, lmbda0 = lame_parameters(req.E, req.nu)
        mat_p, _ = material_vector("neo_hookean", {"mu": mu0, "lmbda": lmbda0}, dtype=p["nodes"].dtype)
        self.params = {**p, "f": f.reshape(-1), "mat_p": mat_p.to(p["nodes"].device)}
        self.ws.retarget(self.params)
        return self.params

    def close(self):
        if self.ws.pcg is not None:
            self.ws.pcg.close()
        if self.ws.mg is not None:
            self.ws.mg.close()


class WorkspacePool:
    """
    Idle ``PooledSolve`` entries by (mesh, solver configuration), least recently used first out, within a
    byte budget (device memory the idle entries hold, beside the engine's admission budget).  Thread-safe:
    a slot takes an entry for the length of one solve and gives it back; two requests on one mesh in
    flight at once each get their own entry.
    """

    def __init__(self, budget_bytes):
        from collections import OrderedDict
        self.budget = int(budget_bytes)
        self._idle = OrderedDict()           # key -> [PooledSolve]
        self._bytes = 0
        self._lock = threading.Lock()
        self.hits = self.misses = self.evictions = 0

    def take(self, key):
        with self._lock:
            entries = self._idle.get(key)
            if entries:
                entry = entries.pop()
                if not entries:
                    del self._idle[key]
                self._bytes -= entry.nbytes
                self.hits += 1
                return entry
            self.misses += 1
            return None

    def give(self, key, entry):
        drop = []
        with self._lock:
            if entry.nbytes > self.budget:
                drop.append(entry)
            else:
                while self._bytes + entry.nbytes > self.budget and self._idle:
                    old_key, entries = next(iter(self._idle.items()))
                    victim = entries.pop(0)
                    if not entries:
                        del self._idle[old_key]
                    self._bytes -= victim.nbytes
                    self.evictions += 1
                    drop.append(victim)
                self._idle.setdefault(key, []).append(entry)
                self._idle.move_to_end(key)
                self._bytes += entry.nbytes
        for e in drop:
            e.close()

    @property
    def idle_bytes(self):
        return self._bytes

    def clear(self):
        with self._lock:
            entries = [e for es in self._idle.values() for e in es]
            self._idle.clear()
            self._bytes = 0
        for e in entries:
            e.close()


def solve_request(req, device, precision="fp32", n_load_steps=1, tol_rel=1e-10, pcg_max_iter=5000, pcg_graph=2,
                  host_params=None, pcg_form="auto", fp32_moduli="ref", max_blocks=0,
                  preconditioner="jacobi", batch=None, driver="native", max_newton=25, max_cutbacks=8, pool=None,
                  mg_graphs=True, mg_bounds_every=0, mg_gather=False):
    """
    Build (or copy from ``host_params``) and solve one request on the current stream; returns
    (u on device, info).  ``pcg_graph`` is the PCG launch form (2: unrolled graph, the default for
    a request solved alone; 1: conditional-loop graph; 0: direct launches, the serving engine's default); ``pcg_form`` the product form inside
    it ("auto", "colour" or "gather", see DevicePCG and workspace.pcg_form_for); ``fp32_moduli`` the FP32
    operator's moduli ("ref": reference frame, no gradients read; "physical"); ``max_blocks`` the most blocks
    per PCG launch (0: the whole GPU); ``preconditioner`` "jacobi", "block_jacobi", "multigrid" or "auto"
    (``preconditioner_for``); ``batch`` a ``BatchExecutor`` that runs the PCG solves of all slots together;
    ``driver`` the Newton loop: "native" (the library's C++ driver, one call per solve) or "python"; ``pool`` a
    ``WorkspacePool`` that keeps the mesh and workspace of a solved request for the next request on the same
    mesh (not used with ``host_params``, whose dictionary the caller built); ``mg_graphs`` the multigrid
    hierarchy's graph-driven mode (see multigrid.Multigrid).  The request is validated on the host first
    (``Request.validate``).
    """
    req.validate()
    preconditioner = preconditioner_for(req, preconditioner)
    if preconditioner == "multigrid":
        batch = None                     # the multigrid PCG runs per request (host-driven, graph-replayed cycle)
    if batch is not None:
        pool = None                      # workspaces bound to a batch executor are not kept
    key = (req.element_type, req.nx, precision, preconditioner, pcg_form, fp32_moduli, max_blocks, pcg_graph,
           mg_graphs, mg_bounds_every, mg_gather, str(device)) if (pool is not None and host_params is None) else None
    entry = pool.take(key) if key is not None else None
    if entry is not None:
        p, ws = entry.retarget(req), entry.ws
    else:
        if host_params is not None:
            p = {k: (v.to(device, non_blocking=True) if torch.is_tensor(v) else v) for k, v in host_params.items()}
        else:
            p = request_problem(req, device, build_on_device=True)
        ws = NewtonWorkspace(p, precision, use_graph=pcg_graph, pcg_form=pcg_form, fp32_moduli=fp32_moduli,
                             max_blocks=max_blocks, preconditioner=preconditioner, batch=batch, mg_graphs=mg_graphs,
                             mg_bounds_every=mg_bounds_every, mg_gather=mg_gather)
    th = torch.ones(p["conn"].shape[0], dtype=torch.float64, device=device)
    tol = tol_rel * float(torch.linalg.vector_norm(p["f"]))
    if batch is not None:
        driver = "python"                # the batched PCG is driven from the executor's thread
    try:
        u, info = newton_krylov_solve(p, th, n_load_steps, tol, max_newton=max_newton, verbose=False, workspace=ws,
                                      precision=precision, pcg_max_iter=pcg_max_iter, preconditioner=preconditioner,
                                      driver=driver, max_cutbacks=max_cutbacks)
    except BaseException:
        if entry is not None:
            entry.close()
        raise
    if key is not None:
        pool.give(key, entry if entry is not None else
                  PooledSolve(req, p, ws, hbm_estimate(req, precision, preconditioner)))
    elif ws.pcg is not None:
        ws.pcg.close()
    return u, info


class ServingEngine:
    """
    Slots x worker threads, one CUDA stream each, admission by an HBM budget.  ``run(requests)`` replays
    the requests at their arrival times (relative to the call) and returns one Result per request.
    """

    def __init__(self, n_slots=16, hbm_budget=None, precision="fp32", device=None, n_load_steps=1, tol_rel=1e-10,
                 pcg_max_iter=5000, prewarm_bytes=0, pcg_graph=0, pcg_form="gather",
                 fp32_moduli="ref", order="fifo", max_blocks=64, preconditioner="auto", batched=False,
                 driver="native", max_newton=25, max_cutbacks=8, pool_bytes=0, mg_graphs=False, mg_bounds_every=3,
                 mg_gather=True):
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        if self.device.index is None:            # "cuda": the current device, by index (the slot threads set it)
            self.device = torch.device(self.device.type, torch.cuda.current_device())
        if hbm_budget is None:
            free, _ = torch.cuda.mem_get_info(self.device)
            hbm_budget = int(0.6 * free)
        self.n_slots, self.hbm_budget, self.precision = n_slots, int(hbm_budget), precision
        # pool_bytes > 0 keeps the meshes of served requests for later requests on the same mesh (their
        # workspaces, PCG graphs and multigrid hierarchies) within that much device memory beside the admission
        # budget (None: 20 % of the free memory).  Off by default: on the seeded stream few requests share a
        # mesh (16 % of a 256-request window), and the memory the idle entries hold makes the other requests
        # allocate anew (measured: 80.9 vs 93.8 solves/s with 32 slots).
        # mg_graphs: the multigrid hierarchies' graph-driven mode.  Off by default in the engine: a request's
        # ~6 set-ups do not repay capturing and instantiating its graphs while 31 other slots launch (measured:
        # 59.4 vs 93.8 solves/s), although one request alone is faster with it (54.5 vs 72.9 ms).
        # mg_bounds_every=3: the smoother bounds are estimated at a request's first set-up and every third one
        # after it (measured: 101-113 vs 70-75 solves/s with estimates at every set-up, the same Newton and
        # PCG iteration counts to 0.05 %).  mg_gather: level 0 of the hierarchy in the gather form, whose node pass
        # also does the smoothing update (2 launches per smoothing step instead of 6): 178.5 vs 166.1 solves/s on
        # 320 requests of the stream (medians of three).
        # pcg_graph=0: the Jacobi PCG launches its kernels directly (status read every 16 iterations).  Capturing
        # and instantiating a graph per request made the 32-slot engine stall from run to run (80 small requests:
        # 42-181 solves/s with unrolled graphs, 168-178 with direct launches, 132-139 with the conditional loop);
        # a request served alone keeps solve_request's unrolled graph.
        if pool_bytes is None:
            free, _ = torch.cuda.mem_get_info(self.device)
            pool_bytes = int(0.2 * free)
        self.pool = WorkspacePool(pool_bytes) if pool_bytes > 0 else None
        # batched: the PCG solves of all slots advance together on one stream (BatchExecutor), one set of
        # launches per iteration for all of them
        self.batch = None
        if batched:
            from difffea_b200.krylov import BatchExecutor
            self.batch = BatchExecutor(self.device, capacity=n_slots, max_blocks=max_blocks)
        self.solve_kw = dict(precision=precision, n_load_steps=n_load_steps, tol_rel=tol_rel, pcg_max_iter=pcg_max_iter,
                             pcg_graph=pcg_graph, pcg_form=pcg_form, fp32_moduli=fp32_moduli, max_blocks=max_blocks,
                             preconditioner=preconditioner, batch=self.batch, driver=driver, max_newton=max_newton,
                             max_cutbacks=max_cutbacks, pool=self.pool, mg_graphs=mg_graphs,
                             mg_bounds_every=mg_bounds_every, mg_gather=mg_gather)
        # torch's caching allocator keeps one pool per stream; a slot whose pool already holds a block of
        # the largest request never calls cudaMalloc (which synchronises the whole device) mid-run
        self.prewarm_bytes = int(prewarm_bytes)
        # which waiting request a free slot takes: "fifo" (arrival order) or "largest_first" (the largest
        # waiting request, by HBM footprint: for a backlog this is longest-processing-time-first, which
        # keeps the slots busy until the end instead of leaving one large request running alone)
        if order not in ("fifo", "largest_first"):
            raise ValueError("order must be 'fifo' or 'largest_first'")
        self.order = order
        # slots share the GPU: each PCG launch takes at most this many blocks (of 148 SMs' worth), so that
        # launches of several slots run side by side instead of each spreading thinly over the whole GPU
        # (measured: 23.6 solves/s at 64 blocks vs 19.7 unlimited, 24 slots, 128 requests of the stream)
        self.max_blocks = int(max_blocks)
        # pcg_form "gather" (3 kernels per iteration) rather than the fused form (2): with many solves in
        # flight the fused form's extra gathers (r, M^-1, p at every element node) cost more than the
        # launch it saves (measured: 24.0 vs 20.7 solves/s, 24 slots, 128 requests of the stream)
        self._cv = threading.Condition()
        self._in_use = 0
        self.peak_in_use = 0
        self.peak_in_flight = 0
        self._in_flight = 0

    # admission ------------------------------------------------------------------------------------
    def _reserve(self, nbytes):
        with self._cv:
            if nbytes > self.hbm_budget:
                raise MemoryError(f"request needs {nbytes} B, the HBM budget is {self.hbm_budget} B")
            while self._in_use + nbytes > self.hbm_budget:
                self._cv.wait()
            self._in_use += nbytes
            self._in_flight += 1
            self.peak_in_use = max(self.peak_in_use, self._in_use)
            self.peak_in_flight = max(self.peak_in_flight, self._in_flight)

    def _release(self, nbytes):
        with self._cv:
            self._in_use -= nbytes
            self._in_flight -= 1
            self._cv.notify_all()

    def _slot_streams(self):
        """One stream per slot, created once; each stream's allocator pool is pre-warmed if asked."""
        if getattr(self, "_streams", None) is None:
            self._streams = [torch.cuda.Stream(self.device) for _ in range(self.n_slots)]
            if self.prewarm_bytes > 0:
                for st in self._streams:
                    with torch.cuda.stream(st):
                        blk = torch.empty(self.prewarm_bytes, dtype=torch.uint8, device=self.device)
                        del blk
                torch.cuda.synchronize(self.device)
        return self._streams

    # run --------------------------------------------------------------------------------------------
    def run(self, requests, keep_solutions=True, host_params=None, source="device"):
        """
        Serve ``requests``.  Where a slot gets a request's problem dictionary: ``source="device"`` builds it on
        the GPU (torch ops on the slot's stream); ``source="host"`` builds it on the CPU, pins it and copies it
        to the device inside the slot (the path of a client that submits requests from host memory);
        ``host_params`` (rid -> problem dictionary in pinned host memory) copies a dictionary built before the
        call.  After the call ``self.device_ms`` is the device time from the first slot's start to the last
        slot's end (CUDA events joined over the slot streams) and ``self.wall`` the host wall time.
        """
        if source not in ("device", "host"):
            raise ValueError("source must be 'device' or 'host'")
        results = {r.rid: Result(r.rid, arrival=r.arrival) for r in requests}
        q = queue.PriorityQueue()      # entries (priority, sequence, request); None ends a worker
        streams = self._slot_streams()
        main = torch.cuda.current_stream(self.device)
        ev_start, ev_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev_start.record(main)
        for st in streams:
            st.wait_event(ev_start)
        t0 = time.perf_counter()
        errors = []

        def worker(stream):
            torch.cuda.set_device(self.device)
            while True:
                req = q.get()[2]
                if req is None:
                    return
                res = results[req.rid]
                reserved = False
                try:
                    req.validate()
                    nbytes = hbm_estimate(req, self.precision, self.solve_kw["preconditioner"])
                    self._reserve(nbytes)
                    reserved = True
                    res.admitted = time.perf_counter() - t0
                    with torch.cuda.stream(stream):
                        hp = host_params.get(req.rid) if host_params is not None else None
                        if hp is None and source == "host":
                            hp = request_problem(req, "cpu", pin_memory=True)
                        u, info = solve_request(req, self.device, host_params=hp, **self.solve_kw)
                        res.u = u.to("cpu") if keep_solutions else None
                        stream.synchronize()
                    res.converged, res.newton, res.cg = info["converged"], info["total_newton"], info["total_cg"]
                    res.load_factor = info["load_factor"]
                    if not res.converged:
                        res.error = f"NotConverged: the load continuation stopped at load factor {res.load_factor:g}"
                except Exception as exc:  # a failed request must not take the engine down
                    res.error = f"{type(exc).__name__}: {exc}"
                    errors.append(res.error)
                finally:
                    res.finished = time.perf_counter() - t0
                    if reserved:
                        self._release(nbytes)

        threads = [threading.Thread(target=worker, args=(st,), daemon=True) for st in streams]
        for th in threads:
            th.start()
        seq = 0
        for req in sorted(requests, key=lambda r: r.arrival):
            delay = req.arrival - (time.perf_counter() - t0)
            if delay > 0:
                time.sleep(delay)
            prio = 0
            if self.order == "largest_first":
                try:
                    prio = -hbm_estimate(req, self.precision, self.solve_kw["preconditioner"])
                except (KeyError, ValueError, TypeError):   # a malformed request: its slot reports the error
                    prio = 0
            q.put((prio, seq, req))
            seq += 1
        for _ in threads:
            q.put((math.inf, seq, None))
            seq += 1
        for th in threads:
            th.join()
        for st in streams:
            ev = torch.cuda.Event()
            ev.record(st)
            main.wait_event(ev)
        ev_end.record(main)
        ev_end.synchronize()
        self.device_ms = ev_start.elapsed_time(ev_end)
        self.wall = time.perf_counter() - t0
        return [results[r.rid] for r in requests]


def run_plain(requests, device, precision="fp64", pcg_graph=2, **kw):
    """
    The same requests one after another on one stream -- the plain drop-in path (FP64, the PCG form of
    newton_krylov_solve's default workspace, its Python driver); Results in order.
    """
    kw.setdefault("driver", "python")
    out = []
    t0 = time.perf_counter()
    for req in requests:
        res = Result(req.rid, arrival=0.0)
        res.admitted = time.perf_counter() - t0
        u, info = solve_request(req, device, precision=precision, pcg_graph=pcg_graph, **kw)
        res.u = u.to("cpu")
        res.converged, res.newton, res.cg = info["converged"], info["total_newton"], info["total_cg"]
        res.finished = time.perf_counter() - t0
        out.append(res)
    return out


def percentile(values, q):
    v = sorted(values)
    if not v:
        return math.nan
    k = min(len(v) - 1, max(0, int(math.ceil(q / 100.0 * len(v))) - 1))
    return v[k]


def shard_requests(requests, rank, world):
    """Requests of one replica when ``world`` GPUs serve one stream independently (round robin by id)."""
    return [r for r in requests if r.rid % world == rank]
