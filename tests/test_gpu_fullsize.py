"""The full-size workloads pinned to the reference's own CPU CG.

tests/golden/reference_fullsize_solutions.json holds HiFlow3's lmp CPU
classes' runs (make_fullsize_solutions.py: NAIVE implementation, the exact
CG<LAD> sequence) on the 128^3 Poisson and lognormal-coefficient matrices and
on a stratified sample of 32 systems of the 1,024-system batch, as
iteration counts plus solution fingerprints (problems.solution_probe: norm,
64 Rademacher projections, 2,048 sampled entries).  The device solves are
held to

* FP64 Jacobi-PCG: the reference's iteration count +-1 and the reference's
  converged solution within 1e-10 relative;
* mixed precision (FP32 inner PCG in FP64 refinement, both inner storages):
  the FP64 true residual at the requested tolerance and the error against
  the FP64 CPU CG oracle (the reference run to 1e-13, or 1e-12 for the batch
  systems) no larger than that of the reference's own FP64 CG stopped at the
  same tolerance, times a small factor.
"""
import json
import os

import numpy as np
import pytest

from ba_b200 import lmp
from ba_b200 import problems as P
from ba_b200.batch import Batch

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FIX = json.load(open(os.path.join(GOLD, "reference_fullsize_solutions.json")))
COUNTS = json.load(open(os.path.join(GOLD, "workload_counts.json")))


@pytest.fixture(scope="module")
def plat():
    return lmp.init_platform(0)


@pytest.fixture(scope="module")
def poisson3d():
    return P.poisson_3d(128)


@pytest.fixture(scope="module")
def varcoef3d():
    return P.varcoef_3d(128, 2.0)


def _true_rel_residual(s, x):
    import scipy.sparse as sp
    A = sp.csr_matrix((s.val, s.col, s.rowptr), shape=(s.n, s.n))
    return float(np.linalg.norm(s.b - A @ x) / np.linalg.norm(s.b))


def _fp64_pcg(plat, s, rtol):
    A = lmp.B200_CSR_lMatrix(s.rowptr, s.col, s.val, platform=plat)
    A.tune()
    b = lmp.B200_lVector.from_numpy(s.b, platform=plat)
    x = lmp.B200_lVector.from_numpy(np.zeros(s.n), platform=plat)
    cg = lmp.setup_CG_solver(maxits=20000, atol=0.0, rtol=rtol, dtol=1e8)
    cg.SetupOperator(A)
    st = cg.Solve(b, x)
    return st, cg.iter(), x.numpy()


@pytest.mark.parametrize("name", ["poisson3d_128", "varcoef3d_128"])
def test_fp64_pcg_matches_reference_at_full_size(plat, poisson3d, varcoef3d, name):
    s = poisson3d if name == "poisson3d_128" else varcoef3d
    ref = FIX[f"{name}/jacobi/rtol1e-10"]
    assert (s.n, s.nnz) == (ref["n"], ref["nnz"])
    if name == "poisson3d_128":
        assert ref["iters"] == COUNTS["poisson3d_128/jacobi/rtol1e-10"]["iters"] == 302
    st, iters, x = _fp64_pcg(plat, s, 1e-10)
    assert st == lmp.kSolverSuccess
    assert abs(iters - ref["iters"]) <= 1, (iters, ref["iters"])
    err = P.probe_error(P.solution_probe(x), ref["probe"])
    print(name, "iters", iters, "ref", ref["iters"], "error vs reference", err)
    assert err["proj"] <= 1e-10 and err["sample"] <= 1e-10, err
    assert _true_rel_residual(s, x) <= 1.5e-10


@pytest.mark.parametrize("mode", ["kept", "kept_f64_vectors", "restart"])
def test_mixed_precision_error_vs_cpu_oracle_varcoef3d(plat, varcoef3d, mode):
    """FP32 inner PCG inside FP64 refinement to 1e-10 on the 128^3 sigma = 2
    lognormal matrix -- by default each pass replaces the inner residual by
    the FP64 one every 10x reduction and keeps the search direction; also
    with FP64 inner vectors, and restarted per pass (MPIR's form, inner
    tolerance 1e-5).  The error against the FP64 CPU CG oracle (the reference
    to 1e-13) is held to 10x that of the reference's own FP64 CG stopped at
    1e-10, and the FP64 true residual to the tolerance.  Kept directions stay
    within 1.3x the reference's FP64 iteration count (685); restarts discard
    the Krylov space every pass and take ~1.5x."""
    s = varcoef3d
    oracle13 = FIX["varcoef3d_128/jacobi/rtol1e-13"]["probe"]
    ref_err = P.probe_error(FIX["varcoef3d_128/jacobi/rtol1e-10"]["probe"], oracle13)
    A = lmp.B200_CSR_lMatrix(s.rowptr, s.col, s.val, platform=plat)
    b = lmp.B200_lVector.from_numpy(s.b, platform=plat)
    x = lmp.B200_lVector(s.n, platform=plat)
    m = lmp.MPIR()
    m.SetupOperator(A)
    m.SetInnerStorage(mode == "kept_f64_vectors")
    m.SetInnerRestart(mode == "restart")
    m.SetMpirParameters(0, 40, 0.0, 1e-10, 1e6)
    m.SetLowPrecErrCorSolverParameters(100000, 0.0, 1e-5 if mode == "restart" else 0.1, 1e30)
    assert m.Solve(b, x) == lmp.kSolverSuccess
    xs = x.numpy()
    err = P.probe_error(P.solution_probe(xs), oracle13)
    print(mode, "outer", m.outer_, "inner iters", m.iter(), "error", err, "reference's own", ref_err)
    assert err["proj"] <= 10 * ref_err["proj"] + 1e-12, (err, ref_err)
    assert err["sample"] <= 10 * ref_err["sample"] + 1e-12, (err, ref_err)
    assert _true_rel_residual(s, xs) <= 1.05e-10
    if mode != "restart":
        assert m.iter() <= 1.3 * FIX["varcoef3d_128/jacobi/rtol1e-10"]["iters"], m.iter()


def test_batch_sample_error_vs_cpu_oracle(plat):
    """The stratified sample of 32 systems of the 1,024-system batch,
    solved in one mixed-precision batch to 1e-8; each system's error against
    the reference's FP64 CG to 1e-12 is bounded, and its true residual is at
    the tolerance."""
    rec = FIX["batch1024_sample/jacobi/rtol1e-12"]
    systems = P.batch_systems(1024, sigma=1.0, seed=P.SEED_BATCH)
    pick = P.stratified_sample([s.nnz for s in systems], 32)
    assert pick == rec["indices"]
    sample = [systems[i] for i in pick]
    B = Batch(len(sample), mixed=True, precond=True, rtol=1e-8, platform=plat)
    slots = B.add_many([(s.rowptr, s.col, s.val, s.b) for s in sample])
    B.solve()
    worst = 0.0
    for i, s, r in zip(pick, sample, B.results(slots)):
        ref = rec["systems"][str(i)]
        assert (s.n, s.nnz) == (ref["n"], ref["nnz"])
        assert r.solver_state == lmp.kSolverSuccess, (s.name, r)
        assert _true_rel_residual(s, r.x) <= 1.001e-8, s.name
        err = P.probe_error(P.solution_probe(r.x), ref["probe"])
        worst = max(worst, err["sample"], err["proj"])
    print("batch sample worst error vs FP64 CPU CG oracle", worst)
    assert worst < 1e-6, worst
    B.close()
