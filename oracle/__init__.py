"""CPU oracle for the PCG hot path -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs import
this package, as the checker (and, in bench.py, as the timed CPU reference).
The product library ba_b200 never imports it.

Two checkers:
* ``liboracle.so``: the C restatement in pcg_oracle.c (CG<LAD>, lmp cg(),
  IterateControl, CSR SpMV, BLAS-1, Jacobi, MPIR-style refinement, the
  stationary Jacobi<LAD> solver, BiCGSTAB<LAD> and GMRES<LAD>);
* ``_ref/libhiflow_lmp_ref.so``: HiFlow3's own lmp CPU sources (NAIVE and
  OPENMP implementations, lPreconditioner_Jacobi, lmp cg()) compiled by
  oracle/ref/Makefile, with a driver restating CG<LAD>, Jacobi<LAD>,
  BiCGSTAB<LAD> and GMRES<LAD> over those objects.
"""
from .oracle import (  # noqa: F401
    CTRL_FAIL_DIV,
    CTRL_FAIL_MAXITS,
    CTRL_ITERATE,
    CTRL_SUCCESS_ABS,
    CTRL_SUCCESS_REL,
    IMPL_NAIVE,
    IMPL_OPENMP,
    JACOBI_SMOOTH_DAMPED,
    JACOBI_SMOOTH_NORMAL,
    JACOBI_SOLVE_DAMPED,
    JACOBI_SOLVE_NORMAL,
    OracleResult,
    RefSystem,
    bicgstab,
    cg,
    coo_to_csr,
    dot,
    gmres,
    invdiag,
    iterate_check,
    jacobi,
    lmp_cg,
    mpcg_kept,
    mpir,
    mpir_generic,
    ref_available,
    ref_bicgstab,
    ref_cg,
    ref_coo_to_csr,
    ref_gmres,
    ref_jacobi,
    ref_lmp_cg,
    ref_spmv,
    spmv,
    spmv_nodiag,
)
