"""
Device-resident mesh: the colour-sorted structure-of-arrays layout the kernels read.

``cuda_mesh(params)`` turns a problem dictionary (built by this package or by the reference) into a
``CudaMesh``: it colours the elements on the host (no two elements of a colour share a node), sorts
them by colour and packs connectivity (+ Dirichlet fix bits), cached geometry and original element
ids into SoA arrays on the GPU.  The handle is cached per (conn, dN_dX, w_detJ, m) tensor identity,
so building closures once per Newton step costs nothing after the first call.  Problem dictionaries
are treated as immutable, as in the reference (operators.py:97-120).

HBM layout per element (FP64): conn 4 B x nen, orig 4 B, dN/dX 16 B x nen x n_q, w detJ 8 B x n_q;
per node: one fix-bit byte.  Rows are padded to a multiple of 32 elements.
"""
import ctypes
import weakref

import numpy as np
import torch

from difffea_b200 import _lib
from difffea_b200.elements import default_rule, element_quadrature, quadrature_gradients

_SUPPORTED = {(4, 4): "quad4", (9, 9): "quad9", (3, 1): "tri3", (6, 6): "tri6", (8, 9): "quad8"}


def stream_handle():
    """cudaStream_t of torch's current stream (every launch goes there)."""
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else ctypes.c_void_p(0)


def _require_cuda(*tensors):
    for t in tensors:
        if not (torch.is_tensor(t) and t.is_cuda):
            raise RuntimeError("the difffea_b200 kernels need CUDA tensors (move the problem with "
                               "problem.to_device(params, 'cuda')); there is no CPU path")


def colour_elements(conn_cpu, n_nodes=None):
    """Greedy colouring (C++): (colour (n_el,) int32, n_colours).  Node ids are checked against n_nodes."""
    conn64 = np.ascontiguousarray(conn_cpu.numpy().astype(np.int64))
    n_el, nen = conn64.shape
    if n_nodes is None:
        n_nodes = int(conn64.max()) + 1 if n_el else 1
    colour = np.zeros(n_el, dtype=np.int32)
    nc = ctypes.c_int32(0)
    _lib.call("dfea_colour_elements", conn64.ctypes.data_as(ctypes.c_void_p), n_el, nen, n_nodes,
              colour.ctypes.data_as(ctypes.c_void_p), ctypes.byref(nc))
    return colour, nc.value


class CudaMesh:
    """Colour-sorted SoA mesh on one GPU (see the module docstring)."""

    def __init__(self, params):
        conn, dN, wd, m, nodes = params["conn"], params["dN_dX"], params["w_detJ"], params["m"], params["nodes"]
        _require_cuda(conn, dN, wd, m, nodes)
        n_el, nen = conn.shape
        n_q = dN.shape[1]
        if (nen, n_q) not in _SUPPORTED:
            raise ValueError(f"element with nen={nen}, n_q={n_q} is not built for the GPU")
        if dN.shape != (n_el, n_q, nen, 2) or wd.shape != (n_el, n_q):
            raise ValueError("dN_dX / w_detJ do not match conn")
        N = nodes.shape[0]
        if m.shape != (2 * N,):
            raise ValueError("mask m must have 2N entries")
        if not bool(((m == 0) | (m == 1)).all()):
            raise ValueError("the Dirichlet mask m must hold 0.0 / 1.0 entries")
        self.device = conn.device
        self.element_type = _SUPPORTED[(nen, n_q)]
        self.n_el, self.nen, self.n_q, self.n_nodes = n_el, nen, n_q, N

        colour, nc = colour_elements(conn.detach().cpu(), N)
        order = np.argsort(colour, kind="stable")
        counts = np.bincount(colour, minlength=nc) if n_el else np.zeros(1, dtype=np.int64)
        begin = np.zeros(nc + 1, dtype=np.int64)
        begin[1:] = np.cumsum(counts)
        self.n_colours = nc
        self.colour_begin = begin.tolist()
        self.colour_of_slot = colour[order]
        self.stride = max(32, (n_el + 31) // 32 * 32)
        S = self.stride

        dev = self.device
        self.perm_host = order.astype(np.int64)          # packed slot -> element, on the host
        self.perm = torch.from_numpy(self.perm_host).to(dev)
        self.conn = torch.empty(nen * S, dtype=torch.int32, device=dev)
        self.orig = torch.empty(S, dtype=torch.int32, device=dev)
        self.grad = torch.empty(n_q * nen * S * 2, dtype=torch.float64, device=dev)
        self.wdet = torch.empty(n_q * S, dtype=torch.float64, device=dev)
        self.node_fix = torch.empty(N, dtype=torch.uint8, device=dev)
        self.grad32 = None
        src = [t.detach().to(dev).contiguous() for t in (conn.to(torch.int64), dN.to(torch.float64),
                                                           wd.to(torch.float64), m.to(torch.float64))]
        with torch.cuda.device(dev):
            _lib.call("dfea_mesh_pack", n_el, S, nen, n_q, N, ptr(self.perm), ptr(src[0]), ptr(src[1]),
                      ptr(src[2]), ptr(src[3]), ptr(self.conn), ptr(self.orig), ptr(self.grad), ptr(self.wdet),
                      ptr(self.node_fix), stream_handle())
            # the pack launch is asynchronous and reads `src`: finish it before the copies go away
            # (holding them would also keep the cache key alive)
            torch.cuda.current_stream().synchronize()
        del src
        self.view = _lib.MeshView()
        v = self.view
        v.n_el, v.stride, v.n_nodes = n_el, S, N
        v.nen, v.n_q, v.n_colours, v.reserved = nen, n_q, nc, 0
        for i, b in enumerate(self.colour_begin):
            v.colour_begin[i] = b
        v.conn, v.orig, v.grad, v.wdet = (self.conn.data_ptr(), self.orig.data_ptr(), self.grad.data_ptr(),
                                          self.wdet.data_ptr())
        v.grad32 = None
        v.node_fix = self.node_fix.data_ptr()
        v.node_elem_ptr = None
        v.node_elem = None
        self.node_elem_ptr = self.node_elem = None
        # reference shape gradients at the Gauss points (host values in the view) and, built on demand,
        # the inverse element Jacobians of the reference-frame FP32 operator
        GP = params.get("GP")
        if GP is None or (GP.dtype == torch.float64 and default_rule(self.element_type, GP)):
            GP = element_quadrature(self.element_type)[0]          # the same points, on the host (shared)
        else:
            GP = GP.detach().to("cpu", torch.float64)
        self.ref_grad = quadrature_gradients(self.element_type, GP).to(torch.float64)  # (n_q, nen, 2), host
        flat = self.ref_grad.reshape(-1).tolist()
        for i, x in enumerate(flat):
            v.ref_grad[i] = x
        v.jinv = None
        self.jinv = None
        self._nodes = params["nodes"]
        self._reduce_work = None

    # -------------------------------------------------------------------------------------------
    @property
    def view_ref(self):
        return ctypes.byref(self.view)

    @property
    def n_dof(self):
        return 2 * self.n_nodes

    def ensure_grad32(self):
        """Build the FP32 copy of the gradients (the geometry of the FP32 inner operator) once."""
        if self.grad32 is None:
            self.grad32 = torch.empty(self.n_q * self.nen * self.stride * 2, dtype=torch.float32, device=self.device)
            with torch.cuda.device(self.device):
                _lib.call("dfea_mesh_grad_to_f32", self.view_ref, ptr(self.grad32), stream_handle())
            self.view.grad32 = self.grad32.data_ptr()
        return self.grad32

    def ensure_node_incidence(self):
        """
        Build the node -> element incidence of the gather form once: the slots of node n are the flat
        indices a * stride + e of its (element, local node) pairs, in increasing order.
        """
        if self.node_elem is None:
            S, nen, n, N, dev = self.stride, self.nen, self.n_el, self.n_nodes, self.device
            if nen * S >= 2 ** 31:
                raise ValueError("mesh too large for 32-bit incidence indices")
            i32 = dict(dtype=torch.int32, device=dev)
            ptr_, inc, work = torch.empty(N + 1, **i32), torch.empty(max(nen * n, 1), **i32), torch.empty(N, **i32)
            with torch.cuda.device(dev):
                _lib.call("dfea_mesh_node_incidence", self.view_ref, ptr(ptr_), ptr(inc), ptr(work), stream_handle())
            self.node_elem = inc[:nen * n]
            self.node_elem_ptr = ptr_
            self.view.node_elem_ptr = self.node_elem_ptr.data_ptr()
            self.view.node_elem = self.node_elem.data_ptr()
        return self.node_elem_ptr, self.node_elem

    def ensure_ref_frame(self):
        """
        Inverse element Jacobians Jinv = (dX/dxi)^-1 at the Gauss points, packed [n_q][2][stride] (rows of
        Jinv as f64 pairs), for the reference-frame FP32 operator.  The problem's dN/dX must equal
        Jinv^T dN/dxi with this package's quadrature; a mismatch raises instead of computing a wrong
        operator.
        """
        if self.jinv is None:
            dev, S, nq = self.device, self.stride, self.n_q
            nodes = self._nodes.detach().to(dev, torch.float64).contiguous()
            jinv = torch.empty(nq * 2 * S * 2, dtype=torch.float64, device=dev)
            check = torch.empty(2, dtype=torch.float64, device=dev)
            with torch.cuda.device(dev):
                _lib.call("dfea_mesh_ref_frame", self.view_ref, ptr(nodes), ptr(jinv), ptr(check), stream_handle())
            diff, scale = check.tolist()
            if self.n_el and diff > 1e-9 * scale:
                raise ValueError("dN_dX does not match this package's reference gradients and quadrature; "
                                 "the reference-frame operator cannot be used for this problem")
            self.jinv = jinv.view(nq, 2, S, 2)
            self.view.jinv = self.jinv.data_ptr()
        return self.jinv

    def moduli_numel_ref(self):
        """FP32 entries of the reference-frame moduli (10 per Gauss point)."""
        return self.n_q * 10 * self.stride

    def reduce_work(self):
        if self._reduce_work is None:
            nbytes = int(_lib.load().dfea_reduce_work_bytes(self.view_ref))
            self._reduce_work = torch.zeros(nbytes, dtype=torch.uint8, device=self.device)
        return self._reduce_work

    def moduli_numel(self, dtype=torch.float64):
        return self.n_q * 16 * self.stride

    def hbm_bytes(self):
        t = [self.conn, self.orig, self.grad, self.wdet, self.node_fix, self.perm]
        for extra in (self.grad32, self.node_elem_ptr, self.node_elem, self.jinv):
            if extra is not None:
                t.append(extra)
        return sum(x.numel() * x.element_size() for x in t)


# id(conn) -> [(weakrefs of (conn, dN_dX, w_detJ, m), CudaMesh)].  Keyed by identity (tensors compare
# element-wise, so they cannot be dictionary keys themselves); an entry dies with its conn tensor.
_CACHE = {}


def cuda_mesh(params):
    """The (cached) CudaMesh of a problem dictionary."""
    key_objs = (params["conn"], params["dN_dX"], params["w_detJ"], params["m"])
    k = id(key_objs[0])
    entries = _CACHE.get(k, [])
    for refs, mesh in entries:
        if all(r() is o for r, o in zip(refs, key_objs)):
            return mesh
    mesh = CudaMesh(params)
    entries = [(rf, me) for rf, me in entries if all(r() is not None for r in rf)]
    entries.append((tuple(weakref.ref(o) for o in key_objs), mesh))
    if k not in _CACHE:
        weakref.finalize(key_objs[0], _CACHE.pop, k, None)
    _CACHE[k] = entries
    return mesh
