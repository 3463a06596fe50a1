"""
oracle -- TEST INFRASTRUCTURE, not part of the product.

A CPU restatement (PyTorch CPU, float64) of the reference difffea algorithm for the matrix-free
Newton-Krylov path, used only as the checker: by tests/, by __graft_entry__.smoke() and by bench.py's
cpu_baseline / --impl reference leg.  The product (differentiable-fea_b200/difffea_b200) never imports
it.  Every function cites the reference file:line it restates.  It is pinned against golden vectors
that tests/golden/make_golden.py generated by running the reference itself (tests/test_oracle_golden.py).
"""
from oracle.reference_path import *  # noqa: F401,F403
