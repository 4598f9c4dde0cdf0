"""ba_b200: B200-native (sm_100a) CSR/SELL SpMV and fused BLAS-1 for HiFlow3's
Jacobi-preconditioned CG path, behind a C ABI (include/b200la.h) and a
host-side mirror of the reference's lmp / linear_solver interface (lmp.py)."""
from ._lib import B200LAError, load  # noqa: F401

__all__ = ["B200LAError", "load"]
