"""
The allocation-free PCG entry point (dfea_pcg_solve_noalloc) against the regular device PCG.

dfea_pcg_solve_noalloc serves callers that cannot allocate GPU memory -- for example a solver plugged
into a host application whose memory manager owns the device, or a latency-critical loop in which
cudaMalloc/cudaFree would block or synchronise.  It keeps its Krylov vectors in a fixed scratch array
inside the library instead of a caller buffer.  This file checks, through the C ABI, that two calls in a
row return the same solution and iteration count as dfea_pcg_create/dfea_pcg_solve -- for FP64 vectors and
moduli, FP32 moduli on FP64 vectors (DFEA_MIXED) and FP32 throughout (DFEA_F32, whose Krylov vectors take
half the scratch bytes per node) -- and that a mesh larger than the scratch limit is refused with a clear
error.  The file name sorts last so that pytest collects it after every other test file: a run that stops
at the first failure (-x) has then already run the rest of the suite if this newer entry point fails.  The
tests themselves depend on no other test and pass alone in a fresh process.
"""
import ctypes

import pytest
import torch

from difffea_b200 import _lib
from difffea_b200.cuda_mesh import ptr, stream_handle
from difffea_b200.krylov import DevicePCG
from difffea_b200.operators import make_A_operator_cuda
from difffea_b200.problem import build_rectangle_problem
from golden_utils import rel

pytestmark = pytest.mark.gpu
DEV = "cuda"


def _system(nx, ny, seed=11):
    p = build_rectangle_problem("quad4", nx, ny, float(nx), float(ny), load=(1e-3, 0.0), device=DEV)
    g = torch.Generator().manual_seed(seed)
    n = p["f"].shape[0]
    u = (((torch.rand(n, dtype=torch.float64, generator=g) * 2 - 1) * 0.04).to(DEV)) * p["m"]
    th = torch.exp(0.3 * torch.randn(p["conn"].shape[0], dtype=torch.float64, generator=g)).to(DEV)
    b = (torch.randn(n, dtype=torch.float64, generator=g).to(DEV)) * p["m"]
    A = make_A_operator_cuda(u, th, p)        # kernel (a): moduli and Jacobi diagonal
    A._u, A._theta, A._params = u, th, p
    return A, b


def _noalloc(A, C, diag, b, x, code, rtol, max_iter):
    iters, status = ctypes.c_int32(-1), ctypes.c_int32(-1)
    rc = _lib.load().dfea_pcg_solve_noalloc(A.mesh.view_ref, ptr(C), ptr(diag), ptr(b), ptr(x), code,
                                            rtol, max_iter, ctypes.byref(iters), ctypes.byref(status),
                                            stream_handle())
    return rc, iters.value, status.value


# (vector dtype code, moduli precision, vector dtype, rtol): FP32 vectors stop at a tolerance FP32 can reach
CASES = {"f64": (_lib.DFEA_F64, "fp64", torch.float64, 1e-10),
         "mixed": (_lib.DFEA_MIXED, "fp32", torch.float64, 1e-10),
         "f32": (_lib.DFEA_F32, "fp32", torch.float32, 1e-5)}


@pytest.mark.parametrize("case", sorted(CASES))
def test_noalloc_pcg_matches_the_allocating_pcg_on_two_calls_in_a_row(case):
    code, precision, vt, rtol = CASES[case]
    A64, b = _system(60, 30)
    A = A64 if precision == "fp64" else make_A_operator_cuda(A64._u, A64._theta, A64._params, precision="fp32")
    diag, bb = A64.diag.to(vt).contiguous(), b.to(vt).contiguous()
    x_ref = torch.empty_like(bb)
    solver = DevicePCG(A.mesh, A.C, diag, bb.clone(), x_ref)       # the allocating entry point, same dtypes
    k_ref, status_ref = solver.solve(rtol, 2000)
    assert status_ref == "converged"
    for _ in range(2):                                   # the shared scratch keeps the previous call's contents
        x = torch.full_like(bb, float("nan"))
        rc, k, status = _noalloc(A, A.C, diag, bb, x, code, rtol, 2000)
        assert rc == 0, _lib.last_error()
        assert status == 1 and k == k_ref
        assert rel(x, x_ref) < 1e-12                     # same kernels, same order: the same iterates
    solver.close()


def test_noalloc_pcg_refuses_meshes_beyond_its_scratch():
    A, b = _system(400, 400)                             # 160,801 nodes > DFEA_NOALLOC_MAX_NODES
    x = torch.empty_like(b)
    rc, _, _ = _noalloc(A, A.C, A.diag, b, x, _lib.DFEA_F64, 1e-8, 10)
    assert rc == 1
    assert "exceed" in _lib.last_error()
