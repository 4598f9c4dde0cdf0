"""Mixed-precision refinement (FP32 Jacobi-PCG inside FP64 refinement) on the
GPU against the FP64 CPU oracle: the FP64 residual reaches the stated
tolerance, and the solution's error against the oracle's FP64 CG solution is
reported and bounded."""
import numpy as np
import pytest

import oracle
from ba_b200 import lmp
from ba_b200 import problems as P

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def plat():
    return lmp.init_platform(0)


def _solve_mp(plat, s, rtol, inner_rtol=1e-5, max_outer=20):
    A = lmp.B200_CSR_lMatrix(s.rowptr, s.col, s.val, platform=plat)
    b = lmp.B200_lVector.from_numpy(s.b, platform=plat)
    x = lmp.B200_lVector(s.n, platform=plat)
    m = lmp.MPIR()
    m.SetupOperator(A)
    m.SetMpirParameters(0, max_outer, 0.0, rtol, 1e6)
    m.SetLowPrecErrCorSolverParameters(100000, 0.0, inner_rtol, 1e30)
    st = m.Solve(b, x)
    return st, m, x.numpy()


@pytest.mark.parametrize("case", [("2d", 2, 48, 1.0), ("3d", 3, 20, 2.0), ("2d_s2", 2, 64, 2.0)])
def test_mp_reaches_fp64_tolerance(plat, case):
    _, dim, n, sigma = case
    s = P.q1_system(dim, n, 77 + n, sigma)
    rtol = 1e-10
    st, m, x = _solve_mp(plat, s, rtol)
    assert st == lmp.kSolverSuccess, (m.state_, m.res_rel_)
    assert m.res_rel_ < rtol
    # the reported residual is the true FP64 residual of the returned x; at
    # ~1e-12 a residual evaluation carries ~eps*|A||x| of rounding, so two
    # evaluations (device FMA rows vs the oracle's loop) agree to a few percent
    r = s.b - oracle.spmv(s.rowptr, s.col, s.val, x)
    floor = 32 * np.finfo(float).eps * np.linalg.norm(oracle.spmv(s.rowptr, s.col, np.abs(s.val), np.abs(x)))
    assert abs(np.linalg.norm(r) - m.res()) <= 0.05 * m.res() + floor
    assert np.linalg.norm(r) < rtol * np.linalg.norm(s.b) * 1.05
    # error against the FP64 oracle's converged CG solution
    ref = oracle.cg(s.rowptr, s.col, s.val, s.b, maxits=100000, atol=0.0, rtol=1e-13)
    err = np.linalg.norm(x - ref.x) / np.linalg.norm(ref.x)
    assert err < 1e-7, err
    # structure: a few FP32 passes, like the oracle's MPIR restatement
    omp, outer = oracle.mpir(s.rowptr, s.col, s.val, s.b, rtol=rtol, inner_rtol=1e-5)
    assert omp.state == 0
    assert abs(m.outer_ - outer) <= 1
    assert m.iter() <= 1.5 * omp.iters + 20


def test_mp_1e8_and_zero_rhs(plat):
    s = P.q1_system(2, 40, 5, 1.0)
    st, m, x = _solve_mp(plat, s, 1e-8, inner_rtol=1e-4)
    assert st == lmp.kSolverSuccess and m.res_rel_ < 1e-8
    z = P.q1_system(2, 8, 1, 0.0)
    z.b[:] = 0.0
    st, m, x = _solve_mp(plat, z, 1e-10)
    assert st == lmp.kSolverSuccess and m.outer_ == 0 and not x.any()


def test_mp_pass_limit_reports_exceeded(plat):
    s = P.q1_system(3, 16, 9, 2.0)
    st, m, x = _solve_mp(plat, s, 1e-12, inner_rtol=1e-2, max_outer=2)
    assert st == lmp.kSolverExceeded
    assert m.outer_ == 2
