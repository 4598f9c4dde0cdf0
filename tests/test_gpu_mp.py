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


def _solve_mp(plat, s, rtol, inner_rtol=1e-5, max_outer=20, restart=True):
    A = lmp.B200_CSR_lMatrix(s.rowptr, s.col, s.val, platform=plat)
    b = lmp.B200_lVector.from_numpy(s.b, platform=plat)
    x = lmp.B200_lVector(s.n, platform=plat)
    m = lmp.MPIR()
    m.SetupOperator(A)
    m.SetInnerRestart(restart)
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


@pytest.mark.parametrize("case", [("2d", 2, 48, 1.0), ("3d", 3, 20, 2.0)])
def test_mp_fp32_values_fp64_vectors(plat, case):
    """Mixed storage: FP32 matrix values under FP64 inner vectors and dots.
    Same bars as the FP32 inner solve (FP64 residual at the tolerance, error
    against the converged FP64 oracle), and the inner iteration count of the
    first pass is close to the FP64 PCG's own count to that inner tolerance."""
    _, dim, n, sigma = case
    s = P.q1_system(dim, n, 77 + n, sigma)
    A = lmp.B200_CSR_lMatrix(s.rowptr, s.col, s.val, platform=plat)
    b = lmp.B200_lVector.from_numpy(s.b, platform=plat)
    x = lmp.B200_lVector(s.n, platform=plat)
    m = lmp.MPIR()
    m.SetupOperator(A)
    m.SetInnerStorage(True)
    m.SetInnerRestart(True)
    m.SetMpirParameters(0, 20, 0.0, 1e-10, 1e6)
    m.SetLowPrecErrCorSolverParameters(100000, 0.0, 1e-5, 1e30)
    assert m.Solve(b, x) == lmp.kSolverSuccess
    xs = x.numpy()
    assert np.linalg.norm(s.b - oracle.spmv(s.rowptr, s.col, s.val, xs)) < 1.05e-10 * np.linalg.norm(s.b)
    ref = oracle.cg(s.rowptr, s.col, s.val, s.b, maxits=100000, atol=0.0, rtol=1e-13)
    assert np.linalg.norm(xs - ref.x) / np.linalg.norm(ref.x) < 1e-8
    # first pass against the FP64 PCG to the same inner tolerance
    m1 = lmp.MPIR()
    m1.SetupOperator(A)
    m1.SetInnerStorage(True)
    m1.SetMpirParameters(0, 1, 0.0, 1e-30, 1e6)
    m1.SetLowPrecErrCorSolverParameters(100000, 0.0, 1e-5, 1e30)
    x1 = lmp.B200_lVector(s.n, platform=plat)
    m1.Solve(b, x1)
    r64 = oracle.cg(s.rowptr, s.col, s.val, s.b, maxits=100000, atol=0.0, rtol=1e-5)
    assert m1.outer_ == 1 and abs(m1.iter() - r64.iters) <= max(2, 0.05 * r64.iters), (m1.iter(), r64.iters)


@pytest.mark.parametrize("case", [("2d", 2, 48, 1.0), ("3d", 3, 20, 2.0), ("2d_s2", 2, 64, 2.0), ("3d40", 3, 40, 2.0)])
def test_mp_kept_direction_matches_oracle(plat, case):
    """The default fused refinement: the inner FP32 PCG's residual is
    replaced by the FP64 residual every 10x reduction and its search
    direction kept.  Same passes as the oracle's restatement
    (oracle.mpcg_kept) within one, total inner iterations within 10%, the
    FP64 residual at the tolerance, and fewer iterations than restarting."""
    _, dim, n, sigma = case
    s = P.q1_system(dim, n, 77 + n, sigma)
    st, m, x = _solve_mp(plat, s, 1e-10, inner_rtol=0.1, max_outer=40, restart=False)
    ref, passes = oracle.mpcg_kept(s.rowptr, s.col, s.val, s.b, rtol=1e-10, inner_rtol=0.1, max_outer=40)
    assert st == lmp.kSolverSuccess and ref.state == 0
    assert abs(m.outer_ - passes) <= 1, (m.outer_, passes)
    assert abs(m.iter() - ref.iters) <= max(3, 0.1 * ref.iters), (m.iter(), ref.iters)
    assert np.linalg.norm(s.b - oracle.spmv(s.rowptr, s.col, s.val, x)) < 1.05e-10 * np.linalg.norm(s.b)
    f64 = oracle.cg(s.rowptr, s.col, s.val, s.b, maxits=100000, atol=0.0, rtol=1e-10)
    rst, _ = oracle.mpir(s.rowptr, s.col, s.val, s.b, rtol=1e-10, inner_rtol=1e-5)
    assert m.iter() < rst.iters and m.iter() <= 1.3 * f64.iters, (m.iter(), rst.iters, f64.iters)


def test_mp_pass_limit_reports_exceeded(plat):
    s = P.q1_system(3, 16, 9, 2.0)
    st, m, x = _solve_mp(plat, s, 1e-12, inner_rtol=1e-2, max_outer=2)
    assert st == lmp.kSolverExceeded
    assert m.outer_ == 2


# ---- generic MPIR (mpir.cc:52-297) over the device solvers -------------------------

def _mpir_generic(plat, s, cfg):
    A = lmp.B200_CSR_lMatrix(s.rowptr, s.col, s.val, platform=plat)
    mp = lmp.MPIR()
    mp.SetupOperator(A)
    ecl = lmp.GMRES()
    ecl.InitParameter(30, "RightPreconditioning")
    pc = lmp.PreconditionerBlockJacobiStand()
    pc.Init_Jacobi()
    ecl.SetupPreconditioner(pc)
    ech = lmp.BiCGSTAB()
    ech.SetupPreconditioner(pc)
    prel = lmp.Jacobi()
    prel.SetSolveMode(2)
    prel.SetNumIter(3)
    posth = lmp.Jacobi()
    posth.SetSolveMode(3)
    posth.SetDampingParameter(0.8)
    mp.SetLowPrecErrCorSolver(ecl)
    mp.SetHighPrecErrCorSolver(ech)
    mp.SetLowPrecPreSmoother(prel)
    mp.SetHighPrecPostSmoother(posth)
    mp.UseLowPrecPreSmoother(True)
    mp.UseHighPrecPostSmoother(True)
    mp.SetMpirParameters(cfg["max_ech"], cfg["max_ecl"], cfg["abs_tol"], cfg["rel_tol"], 1e8)
    mp.SetLowPrecErrCorSolverParameters(*cfg["ecl"])
    mp.SetHighPrecErrCorSolverParameters(*cfg["ech"])
    mp.SetLowPrecPreSmootherParameters(*cfg["prel"])
    mp.SetHighPrecPostSmootherParameters(*cfg["posth"])
    b = lmp.B200_lVector.from_numpy(s.b, platform=plat)
    x = lmp.B200_lVector.from_numpy(np.zeros(s.n), platform=plat)
    st = mp.Solve(b, x)
    return mp, st, x.numpy()


@pytest.mark.parametrize("max_ecl,max_ech", [(3, 0), (1, 2), (0, 2)])
def test_generic_mpir_matches_oracle_loop(plat, max_ecl, max_ech):
    s = P.q1_system(2, 40, 3, 1.0, "mp_generic")
    cfg = {"max_ecl": max_ecl, "max_ech": max_ech, "abs_tol": 1e-9, "rel_tol": 1e-14,
           "ecl": (2000, 0.0, 1e-4, 1e8), "ech": (2000, 1e-12, 1e-6, 1e8), "prel": (3, 0.0, 0.0, 1e8),
           "posth": (2, 0.0, 0.0, 1e8)}
    comps = {"ecl": ("gmres", {"precond": True, "size_basis": 30}, cfg["ecl"]),
             "ech": ("bicgstab", {"precond": True}, cfg["ech"]),
             "prel": ("jacobi", {"mode": 2, "smooth_iter": 3}, cfg["prel"]),
             "posth": ("jacobi", {"mode": 3, "w": 0.8}, cfg["posth"])}
    ref = oracle.mpir_generic(s.rowptr, s.col, s.val, s.b, max_ech=max_ech, max_ecl=max_ecl, abs_tol=1e-9,
                              rel_tol=1e-14, div_tol=1e8, components=comps, use={"prel": True, "posth": True})
    mp, st, x = _mpir_generic(plat, s, cfg)
    assert (mp.n_ecl, mp.n_ech, mp.outer_) == (ref["n_ecl"], ref["n_ech"], ref["passes"])
    assert (st == lmp.kSolverSuccess) == ref["success"]
    assert abs(mp.iter() - ref["iters"]) <= max(3, int(0.1 * ref["iters"]))
    true_res = np.linalg.norm(s.b - oracle.spmv(s.rowptr, s.col, s.val, x))
    if ref["success"]:
        assert true_res <= 1e-9 * 1.001
