"""
Device-resident Jacobi-PCG (kernel (c)) bound to fixed buffers.

``DevicePCG`` owns a ``dfea_pcg`` handle: one PCG iteration (the colour passes of the tangent product
with the curvature fused in, two fused vector-update kernels, the loop condition) captured once in a
CUDA graph with a device-side while-loop, so a whole solve is one graph launch and one read-back of
(status, iterations).  The buffers it binds (moduli, diagonal, right-hand side, solution and a work
area for the Krylov vectors and partial sums) stay allocated for the life of the object; their
contents may change between solves.
"""
import ctypes
import os
import queue
import threading
import warnings

import torch

from difffea_b200 import _lib, ops
from difffea_b200.cuda_mesh import ptr, stream_handle


class DevicePCG:
    """
    use_graph: True / 1 (default) the conditional while-loop graph; 2 an unrolled graph of 8 iterations
    replayed until done (no conditional node: overlaps better with other streams, as in serving);
    False / 0 (or DFEA_PCG_GRAPH=0 in the environment) the same kernels launched directly, polled every
    16 iterations -- also the form for profilers that trace individual launches.
    form: "colour" (one launch per colour, scatter by read-modify-write) or "gather" (one element pass,
    per-node sums fused into the first vector update: 3 kernels per iteration; needs the mesh's node
    incidence, built here) or "fused" (the gather form with the direction update moved into the next
    element pass: 2 kernels per iteration).  Each form is reproducible; they agree to rounding.
    moduli: "physical" (C with the packed dN/dX: FP64, FP32, or FP32 on FP64 vectors) or "ref" (FP32
    moduli pulled back to the element reference frame, 10 per Gauss point, FP64 vectors; the product
    reads no gradients).  max_blocks: at most this many blocks per launch (0: the whole GPU), for solves
    that share the GPU with others; results agree with the unlimited form's to rounding.
    preconditioner: "jacobi" (diag = the (2N,) diagonal) or "block_jacobi" (diag = the (4N,) inverse 2x2
    node blocks of dfea_qp_moduli_block; FP64 vectors).
    """

    def __init__(self, mesh, C, diag, b, x, use_graph=True, form="colour", moduli="physical", max_blocks=0,
                 preconditioner="jacobi"):
        use_graph = int(use_graph) if os.environ.get("DFEA_PCG_GRAPH", "1") != "0" else 0
        if form not in ("colour", "gather", "fused"):
            raise ValueError("form must be 'colour', 'gather' or 'fused'")
        flags = 0
        if form in ("gather", "fused"):
            mesh.ensure_node_incidence()
            flags = _lib.DFEA_PCG_GATHER | (_lib.DFEA_PCG_FUSED if form == "fused" else 0)
        flags |= _lib.pcg_max_blocks(max_blocks)
        if preconditioner == "block_jacobi":
            # diag holds the inverse 2x2 node blocks (4N doubles) of dfea_qp_moduli_block
            if diag.dtype != torch.float64 or diag.numel() != 2 * mesh.n_dof or b.dtype != torch.float64:
                raise ValueError("block-Jacobi: diag must be the (4N,) f64 inverse blocks, vectors f64")
            flags |= _lib.DFEA_PCG_BLOCK_JACOBI
        elif preconditioner != "jacobi":
            raise ValueError("preconditioner must be 'jacobi' or 'block_jacobi'")
        self.preconditioner = preconditioner
        vt = b.dtype
        if moduli == "ref":
            # FP32 moduli in the element reference frame (10 per Gauss point): no gradients read
            if C.dtype != torch.float32 or vt != torch.float64 or C.numel() != mesh.moduli_numel_ref():
                raise ValueError("reference-frame moduli: FP32, 10 per Gauss point, with FP64 vectors")
            dt = _lib.DFEA_F32REF
        elif moduli != "physical":
            raise ValueError("moduli must be 'physical' or 'ref'")
        elif C.dtype == torch.float64:
            dt = _lib.DFEA_F64
            if vt != torch.float64:
                raise ValueError("FP64 moduli need FP64 vectors")
        else:
            dt = _lib.DFEA_MIXED if vt == torch.float64 else _lib.DFEA_F32
        n_diag = 2 * mesh.n_dof if preconditioner == "block_jacobi" else mesh.n_dof
        for name, t, n_t in (("diag", diag, n_diag), ("b", b, mesh.n_dof), ("x", x, mesh.n_dof)):
            if t.dtype != vt or t.numel() != n_t or not t.is_contiguous() or t.device != mesh.device:
                raise ValueError(f"{name} must be a contiguous ({n_t},) {vt} tensor on {mesh.device}")
        if dt in (_lib.DFEA_MIXED, _lib.DFEA_F32):
            mesh.ensure_grad32()
        self.mesh, self.C, self.diag, self.b, self.x = mesh, C, diag, b, x
        self.vec_dtype = vt
        nbytes = int(_lib.load().dfea_pcg_work_bytes(mesh.view_ref, dt))
        self.work = torch.empty(nbytes, dtype=torch.uint8, device=mesh.device)
        self._h = ctypes.c_void_p(0)
        with torch.cuda.device(mesh.device):
            # the handle zeroes its work area on an internal stream: order it after torch's stream
            torch.cuda.current_stream().synchronize()
            rc = _lib.load().dfea_pcg_create(mesh.view_ref, ptr(C), ptr(diag), ptr(b), ptr(x), dt, ptr(self.work),
                                             use_graph | flags, ctypes.byref(self._h))
            if rc != _lib.DFEA_OK and use_graph:
                # the conditional-graph path could not be built on this device/driver: same kernels,
                # launched directly (host-polled), rather than failing the solve
                warnings.warn(f"PCG graph unavailable ({_lib.last_error()}); using direct launches")
                use_graph = False
                rc = _lib.load().dfea_pcg_create(mesh.view_ref, ptr(C), ptr(diag), ptr(b), ptr(x), dt,
                                                 ptr(self.work), flags, ctypes.byref(self._h))
            _lib.check(rc, "dfea_pcg_create")
        self.use_graph = use_graph
        self.form = form
        self.last_status = None
        self.id = ops.register_handle(self)

    def solve(self, rtol, max_iter=500):
        """Run PCG on the bound buffers (custom op pcg_solve); returns (iterations, status string).  Blocks
        until done."""
        it, st = torch.ops.difffea_b200.pcg_solve(self.id, self.x, float(rtol), int(max_iter)).tolist()
        self.last_status = _lib.PCG_STATUS.get(st, str(st))
        return it, self.last_status

    def close(self):
        if self._h and self._h.value:
            _lib.load().dfea_pcg_destroy(self._h)
            self._h = ctypes.c_void_p(0)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class _Ticket:
    __slots__ = ("pcg", "rtol", "max_iter", "event", "done", "iters", "status", "error", "rounds")

    def __init__(self, pcg, rtol, max_iter, event):
        self.pcg, self.rtol, self.max_iter, self.event = pcg, rtol, max_iter, event
        self.done = threading.Event()
        self.iters, self.status, self.error, self.rounds = 0, None, "", 0


class BatchExecutor:
    """
    Runs the PCG solves of many threads together on one stream: every round advances all solves in
    flight by ``iterations_per_check`` iterations with one element-pass launch per element type and one
    launch of each vector update for all of them (``dfea_batch_*``), then reads their statuses.  A
    thread calls ``solve(pcg, rtol, max_iter)`` after queueing the right-hand side on its current
    stream; the call returns when that solve has ended (its ``x`` is then final).  New solves join at
    the next round.  Each solve's iterates are bitwise those of ``pcg.solve`` alone (same block cap).
    Handles must be in the serving configuration: gather form, Jacobi, reference-frame FP32 moduli.
    """

    def __init__(self, device, capacity=64, max_blocks=64, iterations_per_check=8):
        device = torch.device(device)
        if device.index is None:
            device = torch.device("cuda", torch.cuda.current_device())
        self.device = device
        self.capacity, self.max_blocks, self.iterations_per_check = int(capacity), int(max_blocks), int(iterations_per_check)
        self._h = ctypes.c_void_p(0)
        with torch.cuda.device(self.device):
            _lib.call("dfea_batch_create", self.capacity, self.max_blocks, ctypes.byref(self._h))
            self.stream = torch.cuda.Stream(self.device)
        self._q = queue.Queue()
        self._failure = ""
        self.rounds = 0
        self.peak_batch = 0
        self._thread = threading.Thread(target=self._loop, daemon=True)
        self._thread.start()

    def solve(self, pcg, rtol, max_iter):
        ev = torch.cuda.Event()
        ev.record(torch.cuda.current_stream(self.device))
        t = _Ticket(pcg, float(rtol), int(max_iter), ev)
        self._q.put(t)
        while not t.done.wait(1.0):
            if not self._thread.is_alive():   # the executor ended: this solve will never be served
                raise RuntimeError(f"batch executor stopped: {self._failure or 'closed'}")
        if t.error:
            raise RuntimeError(t.error)
        pcg.last_status = t.status
        return t.iters, t.status

    def _set(self, active):
        arr = (ctypes.c_void_p * max(1, len(active)))(*[t.pcg._h.value for t in active])
        _lib.call("dfea_batch_set", self._h, arr, len(active), ctypes.c_void_p(self.stream.cuda_stream))

    def _loop(self):
        try:
            self._serve()
        except BaseException as exc:  # anything outside a round: record it, solve() reports it
            self._failure = f"{type(exc).__name__}: {exc}"

    def _serve(self):
        torch.cuda.set_device(self.device)
        status = (ctypes.c_int32 * self.capacity)()
        iters = (ctypes.c_int32 * self.capacity)()
        s = ctypes.c_void_p(self.stream.cuda_stream)
        active, stop = [], False
        while not (stop and not active):
            new = []
            if not active:
                t = self._q.get()
                if t is None:
                    break
                new.append(t)
            while len(active) + len(new) < self.capacity:
                try:
                    t = self._q.get_nowait()
                except queue.Empty:
                    break
                if t is None:
                    stop = True
                    break
                new.append(t)
            try:
                for t in new:
                    self.stream.wait_event(t.event)          # the right-hand side is ready on the caller's stream
                    _lib.call("dfea_batch_start", self._h, t.pcg._h, t.rtol, t.max_iter, s)
                if new:
                    active += new
                    self._set(active)
                self.peak_batch = max(self.peak_batch, len(active))
                _lib.call("dfea_batch_iterate", self._h, self.iterations_per_check, status, iters, s)
                self.rounds += 1
                keep = []
                for i, t in enumerate(active):
                    t.rounds += 1
                    if status[i] != 0:
                        t.iters, t.status = int(iters[i]), _lib.PCG_STATUS.get(status[i], str(status[i]))
                        t.done.set()
                    elif t.rounds * self.iterations_per_check > t.max_iter + 2 * self.iterations_per_check + 8:
                        # the device stops every solve at max_iter; a solve still running is a fault
                        t.error = "batched PCG solve did not end after max_iter iterations"
                        t.done.set()
                    else:
                        keep.append(t)
                if len(keep) != len(active):
                    active = keep
                    self._set(active)
            except Exception as exc:  # a failed round fails its solves, not the executor
                for t in active + new:
                    if not t.done.is_set():
                        t.error = f"{type(exc).__name__}: {exc}"
                        t.done.set()
                active = []

    def close(self):
        if self._thread.is_alive():
            self._q.put(None)
            self._thread.join()
        if self._h and self._h.value:
            _lib.load().dfea_batch_destroy(self._h)
            self._h = ctypes.c_void_p(0)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
