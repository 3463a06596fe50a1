"""
difffea_b200 -- the matrix-free Newton-Krylov hot path of difffea on NVIDIA B200 (sm_100a).

A drop-in ``cuda`` tangent variant for difffea's functional API: problem dictionaries, residual and
tangent-operator closures, the Newton-Krylov solve and the adjoint sensitivity, backed by hand-written
CUDA kernels in libdifffea_b200.so (C ABI: include/difffea_b200.h) and exposed as torch custom ops.
"""
from difffea_b200 import _lib  # noqa: F401

__version__ = "0.1.0"
