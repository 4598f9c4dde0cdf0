"""GPU parity of the B200 path against the CPU oracle, through the C ABI.

Mirrors the reference's own tests (tests/lmp_test.cc, tests/cuda_test.cc,
tests/cg_test.cc: 3x3 known answers, tolerance 1e-12) and extends them to the
generated FE systems: iteration counts equal to the reference's CG within +-1
(FP64) and solutions within 1e-10 relative of the FP64 oracle.
"""
import json
import os

import numpy as np
import pytest

import oracle
from ba_b200 import lmp
from ba_b200 import problems as P
from ba_b200._lib import FMT_CSR, FMT_SELL, FMT_SELL16, FMT_STENCIL, B200LAError

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
SCHEDULES = ([(FMT_CSR, g) for g in (1, 2, 4, 8, 16, 32)] + [(FMT_SELL, w) for w in (1, 2, 4)]
             + [(FMT_SELL16, w) for w in (1, 2, 4)])

# FP64 SpMV tolerance: the device sums each row with FMA in a different order
# than the oracle's sequential loop; bound by a few ulps of sum |a_ij x_j|.
SPMV_RTOL_F64 = 1e-14
SPMV_RTOL_F32 = 1e-5


@pytest.fixture(scope="module")
def plat():
    return lmp.init_platform(0)


def _mat(plat, s, dtype=np.float64):
    return lmp.B200_CSR_lMatrix(s.rowptr, s.col, s.val, platform=plat, dtype=dtype)


def _vec(plat, a, dtype=np.float64):
    return lmp.B200_lVector.from_numpy(np.asarray(a, dtype), platform=plat, dtype=dtype)


def _abs_rowsum(s, x):
    return np.abs(oracle.spmv(s.rowptr, s.col, np.abs(s.val), np.abs(x)))


def test_lmp_test_spmv_known_answer(plat):
    kat = json.load(open(os.path.join(GOLD, "reference_known_answers.json")))
    s7 = P.lmp_test_3x3()
    for fmt, prm in SCHEDULES:
        A = _mat(plat, s7)
        A.set_format(fmt, prm)
        x = _vec(plat, kat["lmp_test_spmv"]["x"])
        y = x.CloneWithoutContent()
        A.VectorMult(x, y)
        np.testing.assert_array_equal(y.numpy(), kat["lmp_test_spmv"]["y"])


def test_cuda_test_spmv_known_answer(plat):
    kat = json.load(open(os.path.join(GOLD, "reference_known_answers.json")))
    s9 = P.known_answer_3x3()
    A = _mat(plat, s9)
    x = _vec(plat, kat["cuda_test_spmv"]["x"])
    y = x.CloneWithoutContent()
    A.VectorMult(x, y)
    np.testing.assert_allclose(y.numpy(), kat["cuda_test_spmv"]["y"], rtol=0, atol=1e-12)


def test_cg_test_known_answer(plat):
    kat = json.load(open(os.path.join(GOLD, "reference_known_answers.json")))
    s = P.known_answer_3x3()
    for precond in (False, True):
        A = _mat(plat, s)
        b = _vec(plat, s.b)
        x = _vec(plat, np.zeros(3))
        solver = lmp.setup_CG_solver(maxits=100, atol=0.0, rtol=1e-14, dtol=1e8, use_precond=precond)
        solver.SetupOperator(A)
        st = solver.Solve(b, x)
        assert st == lmp.kSolverSuccess
        np.testing.assert_allclose(x.numpy(), kat["cg_test_3x3"]["x"], rtol=0, atol=1e-12)


def _spmv_cases():
    yield P.poisson_2d(16)
    yield P.poisson_2d(100)
    yield P.q1_system(3, 10, 3, 2.0)
    yield P.random_spd(17, 1)
    yield P.random_spd(33, 2, empty_rows=3)
    yield P.random_spd(257, 3, density=0.02, empty_rows=5)
    yield P.random_spd(1, 4)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_spmv_all_schedules_vs_oracle(plat, dtype):
    rtol = SPMV_RTOL_F64 if dtype == np.float64 else SPMV_RTOL_F32
    for s in _spmv_cases():
        xs = P.uniform01(5, s.n, stream=9) - 0.5
        ref = oracle.spmv(s.rowptr, s.col, s.val, xs, dtype=np.float64)
        bound = _abs_rowsum(s, xs) * rtol + 1e-300
        for fmt, prm in SCHEDULES:
            A = _mat(plat, s, dtype)
            A.set_format(fmt, prm)
            x = _vec(plat, xs, dtype)
            y = x.CloneWithoutContent()
            A.VectorMult(x, y)
            err = np.abs(y.numpy().astype(np.float64) - ref)
            assert np.all(err <= bound), (s.name, fmt, prm, float(err.max()))
            # y += A x
            A.VectorMultAdd(x, y)
            err2 = np.abs(y.numpy().astype(np.float64) - 2 * ref)
            assert np.all(err2 <= 2 * bound + 1e-300), (s.name, fmt, prm)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_spmv_nodiag_vs_oracle(plat, dtype):
    # VectorMultNoDiag against the oracle's restatement of the reference loop
    # (every stored entry off the diagonal), including rows without a stored
    # diagonal and empty rows
    rtol = SPMV_RTOL_F64 if dtype == np.float64 else SPMV_RTOL_F32
    for s in _spmv_cases():
        xs = P.uniform01(6, s.n, stream=9) - 0.5
        ref = oracle.spmv_nodiag(s.rowptr, s.col, s.val, xs, dtype=np.float64)
        bound = _abs_rowsum(s, xs) * rtol + 1e-300
        A = _mat(plat, s, dtype)
        x = _vec(plat, xs, dtype)
        y = x.CloneWithoutContent()
        A.VectorMultNoDiag(x, y)
        err = np.abs(y.numpy().astype(np.float64) - ref)
        assert np.all(err <= bound), (s.name, float(err.max()))


def test_blas1_vs_oracle(plat):
    rng = np.random.default_rng(7)
    for n in (1, 2, 3, 5, 31, 1000, 4097, 123457):
        a = rng.standard_normal(n)
        b = rng.standard_normal(n)
        va, vb = _vec(plat, a), _vec(plat, b)
        np.testing.assert_allclose(va.Dot(vb), oracle.dot(a, b), rtol=1e-13, atol=1e-13 * n)
        np.testing.assert_allclose(va.Norm2(), np.sqrt(oracle.dot(a, a)), rtol=1e-13)
        va.Axpy(vb, 0.75)
        np.testing.assert_allclose(va.numpy(), a + 0.75 * b, rtol=1e-15, atol=1e-15)
        va.ScaleAdd(-1.5, vb)
        np.testing.assert_allclose(va.numpy(), -1.5 * (a + 0.75 * b) + b, rtol=1e-14, atol=1e-14)
        va.ElementWiseMult(vb)
        np.testing.assert_allclose(va.numpy(), (-1.5 * (a + 0.75 * b) + b) * b, rtol=1e-14, atol=1e-14)
        va.Scale(2.0)
        vc = va.CloneWithoutContent()
        vc.CopyFrom(va)
        np.testing.assert_array_equal(vc.numpy(), va.numpy())
        v32 = lmp.B200_lVector(n, platform=plat, dtype=np.float32)
        v32.CastFrom(vb)
        np.testing.assert_array_equal(v32.numpy(), b.astype(np.float32))
        # float dot: compensated FP32 accumulation
        a32, b32 = a.astype(np.float32), b.astype(np.float32)
        w1, w2 = _vec(plat, a32, np.float32), _vec(plat, b32, np.float32)
        exact = float(np.dot(a32.astype(np.float64), b32.astype(np.float64)))
        assert abs(w1.Dot(w2) - exact) <= 1e-6 * np.sqrt(n) * (np.abs(a32) @ np.abs(b32)) / n + 1e-6


def test_set_get_values_zero_rows_invdiag(plat):
    s = P.q1_system(2, 6, 1, 1.0)
    A = _mat(plat, s)
    inv = lmp.B200_lVector(s.n, platform=plat)
    A.extract_invdiagelements(inv)
    np.testing.assert_array_equal(inv.numpy(), oracle.invdiag(s.rowptr, s.col, s.val))
    v = lmp.B200_lVector(s.n, platform=plat)
    v.SetValues([3, 0, 7], [1.5, -2.0, 4.0])
    np.testing.assert_array_equal(v.GetValues([0, 3, 7, 1]), [-2.0, 1.5, 4.0, 0.0])
    rows = [8, 9]
    A.ZeroRows(rows, 1.0)
    x = _vec(plat, np.arange(s.n, dtype=np.float64))
    y = x.CloneWithoutContent()
    A.VectorMult(x, y)
    np.testing.assert_array_equal(y.GetValues(rows), [8.0, 9.0])
    with pytest.raises(B200LAError):
        v.GetValues([s.n])


def test_missing_diagonal_is_rejected(plat):
    rowptr = np.array([0, 1, 2], np.int32)
    col = np.array([1, 0], np.int32)
    A = lmp.B200_CSR_lMatrix(rowptr, col, np.array([1.0, 1.0]), platform=plat)
    inv = lmp.B200_lVector(2, platform=plat)
    with pytest.raises(B200LAError) as e:
        A.extract_invdiagelements(inv)
    assert e.value.status == -5
    solver = lmp.setup_CG_solver()
    solver.SetupOperator(A)
    with pytest.raises(B200LAError):
        solver.Solve(_vec(plat, [1.0, 1.0]), _vec(plat, [0.0, 0.0]))


def test_malformed_csr_rejected_on_host(plat):
    with pytest.raises(B200LAError) as e:
        lmp.B200_CSR_lMatrix(np.array([0, 2, 1], np.int32), np.array([0, 1], np.int32), np.ones(2),
                             platform=plat)
    assert e.value.status == -5
    with pytest.raises(B200LAError):
        lmp.B200_CSR_lMatrix(np.array([0, 1, 2], np.int32), np.array([0, 5], np.int32), np.ones(2),
                             platform=plat)


def _golden():
    with open(os.path.join(GOLD, "reference_cg_runs.json")) as f:
        return json.load(f)["cases"]


def _golden_system(name):
    from test_oracle import _system
    return _system(name)


@pytest.mark.parametrize("case", _golden(), ids=lambda c: c["name"])
def test_cg_matches_reference_runs(plat, case):
    """Iteration counts of the reference's CG (+-1 FP64) and solutions within
    1e-10 relative (FP64) / the FP32 oracle's own accuracy (FP32)."""
    s = _golden_system(case["name"])
    for run in case["runs"]:
        dt = np.float64 if run["dtype"] == "f64" else np.float32
        same = oracle.cg(s.rowptr, s.col, s.val, s.b, maxits=20000, atol=0.0, rtol=run["rtol"],
                         dtol=1e8, precond=run["precond"], dtype=dt)
        assert same.iters == run["iters"]
        for fmt, prm in ((FMT_CSR, 4), (FMT_CSR, 16), (FMT_SELL, 1), (FMT_SELL16, 2)):
            A = _mat(plat, s, dt)
            A.set_format(fmt, prm)
            b = _vec(plat, s.b, dt)
            x = _vec(plat, np.zeros(s.n), dt)
            solver = lmp.setup_CG_solver(maxits=20000, atol=0.0, rtol=run["rtol"], dtol=1e8,
                                         use_precond=run["precond"])
            solver.SetupOperator(A)
            st = solver.Solve(b, x)
            assert st == lmp.kSolverSuccess
            xd = x.numpy().astype(np.float64)
            if dt == np.float64:
                assert abs(solver.iter() - run["iters"]) <= 1, (solver.iter(), run["iters"])
                np.testing.assert_allclose(solver.res_init(), run["res_init"], rtol=1e-12)
                assert np.linalg.norm(xd - same.x) <= 1e-10 * np.linalg.norm(same.x)
            else:
                assert abs(solver.iter() - run["iters"]) <= max(2, run["iters"] // 10)
                r = s.b - oracle.spmv(s.rowptr, s.col, s.val, xd)
                assert np.linalg.norm(r) <= 20 * run["rtol"] * np.linalg.norm(s.b)


def test_cg_state_semantics(plat):
    s = P.poisson_2d(16)
    A = _mat(plat, s)
    b = _vec(plat, s.b)
    # maxits exceeded -> kSolverExceeded with iter == maxits
    x = _vec(plat, np.zeros(s.n))
    solver = lmp.setup_CG_solver(maxits=7, atol=0.0, rtol=1e-10)
    solver.SetupOperator(A)
    assert solver.Solve(b, x) == lmp.kSolverExceeded
    assert solver.iter() == 7
    ref = oracle.cg(s.rowptr, s.col, s.val, s.b, maxits=7, atol=0.0, rtol=1e-10)
    np.testing.assert_allclose(x.numpy(), ref.x, rtol=1e-12, atol=1e-14)
    # zero rhs -> success at iteration 0 (res <= atol)
    z = _vec(plat, np.zeros(s.n))
    x = _vec(plat, np.zeros(s.n))
    assert solver.Solve(z, x) == lmp.kSolverSuccess and solver.iter() == 0
    # start from the solution's neighbourhood: res_init is that of b - A x0
    x0 = ref.x.copy()
    x = _vec(plat, x0)
    solver = lmp.setup_CG_solver(maxits=5000, atol=0.0, rtol=1e-10)
    solver.SetupOperator(A)
    solver.Solve(b, x)
    r2 = oracle.cg(s.rowptr, s.col, s.val, s.b, x0=x0, maxits=5000, atol=0.0, rtol=1e-10)
    assert abs(solver.iter() - r2.iters) <= 1
    np.testing.assert_allclose(solver.res_init(), r2.res_init, rtol=1e-12)
    # solver reuse gives identical results (deterministic reductions)
    x1 = _vec(plat, np.zeros(s.n))
    solver.Solve(b, x1)
    it1 = solver.iter()
    x2 = _vec(plat, np.zeros(s.n))
    solver.Solve(b, x2)
    assert solver.iter() == it1
    np.testing.assert_array_equal(x1.numpy(), x2.numpy())


def test_cg_poisson2d_256_full_size(plat):
    """2D Q1 Poisson, 256^2 cells (66,049 DOFs), at rel 1e-10."""
    s = P.poisson_2d(256)
    ref = oracle.cg(s.rowptr, s.col, s.val, s.b, maxits=5000, atol=0.0, rtol=1e-10)
    A = _mat(plat, s)
    A.tune()
    b = _vec(plat, s.b)
    x = _vec(plat, np.zeros(s.n))
    solver = lmp.setup_CG_solver(maxits=5000, atol=0.0, rtol=1e-10, dtol=1e8)
    solver.SetupOperator(A)
    assert solver.Solve(b, x) == lmp.kSolverSuccess
    assert abs(solver.iter() - ref.iters) <= 1
    assert np.linalg.norm(x.numpy() - ref.x) <= 1e-10 * np.linalg.norm(ref.x) * 10


def test_cg_3d_vs_oracle(plat):
    s = P.poisson_3d(40)
    ref = oracle.cg(s.rowptr, s.col, s.val, s.b, maxits=5000, atol=0.0, rtol=1e-10)
    A = _mat(plat, s)
    fmt, prm, us = A.tune()
    b = _vec(plat, s.b)
    x = _vec(plat, np.zeros(s.n))
    solver = lmp.setup_CG_solver(maxits=5000, atol=0.0, rtol=1e-10, dtol=1e8)
    solver.SetupOperator(A)
    assert solver.Solve(b, x) == lmp.kSolverSuccess
    assert abs(solver.iter() - ref.iters) <= 1
    assert np.linalg.norm(x.numpy() - ref.x) <= 1e-10 * np.linalg.norm(ref.x) * 10


def test_full_size_poisson3d_128_properties(plat):
    """128^3 Q1 Poisson (2,146,689 DOFs, 57,066,625 nnz): size-independent
    checks -- SpMV against scipy's CSR product, linearity, and a converged
    true residual."""
    import scipy.sparse as sp
    s = P.poisson_3d(128)
    assert s.n == 2146689 and s.nnz == 57066625
    Ah = sp.csr_matrix((s.val, s.col, s.rowptr), shape=(s.n, s.n))
    A = _mat(plat, s)
    A.tune()
    xs = P.uniform01(3, s.n, stream=1)
    ys = P.uniform01(4, s.n, stream=1)
    x, y = _vec(plat, xs), _vec(plat, ys)
    ax, ay = x.CloneWithoutContent(), x.CloneWithoutContent()
    A.VectorMult(x, ax)
    A.VectorMult(y, ay)
    ref = Ah @ xs
    bound = (abs(Ah) @ np.abs(xs)) * 1e-14
    assert np.all(np.abs(ax.numpy() - ref) <= bound)
    x.Axpy(y, 1.0)
    axy = x.CloneWithoutContent()
    A.VectorMult(x, axy)
    np.testing.assert_allclose(axy.numpy(), ax.numpy() + ay.numpy(), rtol=1e-12, atol=1e-13)
    b = _vec(plat, s.b)
    sol = _vec(plat, np.zeros(s.n))
    solver = lmp.setup_CG_solver(maxits=5000, atol=0.0, rtol=1e-10, dtol=1e8)
    solver.SetupOperator(A)
    assert solver.Solve(b, sol) == lmp.kSolverSuccess
    xs_ = sol.numpy()
    true_res = np.linalg.norm(s.b - Ah @ xs_)
    assert true_res <= 2e-10 * np.linalg.norm(s.b)


def test_sell16_matches_sell_bitwise_and_refuses_far_columns(plat):
    """SELL16 stores (column - row) as int16: same products in the same order
    as SELL, so the results are identical; a column more than 32767 rows away
    is refused with B200LA_ERR_UNSUPPORTED (the tuner then skips SELL16)."""
    s = P.q1_system(3, 20, 31, 1.0)
    xs = np.random.default_rng(3).standard_normal(s.n)
    for dt in (np.float64, np.float32):
        ys = []
        for fmt in (FMT_SELL, FMT_SELL16):
            for w in (1, 2, 4):
                A = _mat(plat, s, dt)
                A.set_format(fmt, w)
                x = _vec(plat, xs, dt)
                y = x.CloneWithoutContent()
                A.VectorMult(x, y)
                ys.append((w, y.numpy()))
        for (w1, a), (w2, b) in zip(ys[:3], ys[3:]):
            np.testing.assert_array_equal(a, b)
    n = 40000
    rowptr = np.arange(n + 1, dtype=np.int32)
    col = np.arange(n, dtype=np.int32)
    col[0] = n - 1                      # row 0 reads column 39999
    A = lmp.B200_CSR_lMatrix(rowptr, col, np.ones(n), platform=plat)
    with pytest.raises(B200LAError) as e:
        A.set_format(FMT_SELL16, 1)
    assert e.value.status == -7
    fmt, _, _ = A.tune()
    assert fmt != FMT_SELL16


@pytest.mark.parametrize("case", ["3x3", "2d", "3d_s1", "spd_empty"])
def test_lmp_cg_entry_matches_reference_lmp_cg(plat, case):
    """lmp.cg(): the reference's own lmp cg() (lmp/solvers/cg.h:93-209) as one
    device solve -- its stop rule norm <= max(rel*norm0, abs) and the 0-based
    index it returns in max_iter -- against that function compiled from the
    reference sources (oracle/_ref) and its restatement (oracle.lmp_cg): the
    same returned index +-1 and the solution within 1e-10 relative; the
    tests/cg_test.cc known answer within 1e-12."""
    s = {"3x3": P.known_answer_3x3, "2d": lambda: P.q1_system(2, 40, 5, 0.0),
         "3d_s1": lambda: P.q1_system(3, 12, 7, 1.0), "spd_empty": lambda: P.random_spd(60, 9, empty_rows=3)}[case]()
    rel = 0.0 if case == "3x3" else 1e-10
    A = _mat(plat, s)
    x = _vec(plat, np.zeros(s.n))
    rc, idx = lmp.cg(x, _vec(plat, s.b), A, rel, 0.0, 100 if case == "3x3" else 5000)
    xs = x.numpy()
    ref = oracle.lmp_cg(s.rowptr, s.col, s.val, s.b, rel_eps=rel, abs_eps=0.0, max_iter=100 if case == "3x3" else 5000)
    assert rc == 0
    if oracle.ref_available():
        real = oracle.ref_lmp_cg(s.rowptr, s.col, s.val, s.b, rel_eps=rel, abs_eps=0.0,
                                 max_iter=100 if case == "3x3" else 5000)
        assert real.iters == ref.iters and np.array_equal(real.x, ref.x)
    if case == "3x3":
        # rel = abs = 0 (as cg_test.cc sets them): the reference iterates until
        # ||r|| is exactly 0 (31 iterations in its arithmetic); only the
        # known answer is the bar here, as in cg_test.cc
        np.testing.assert_allclose(xs, [-0.25, -1.5, -0.75], rtol=0, atol=1e-12)
        return
    assert abs(idx - ref.iters) <= 1, (idx, ref.iters)
    assert np.linalg.norm(xs - ref.x) <= 1e-10 * np.linalg.norm(ref.x)


def _ragged(n, seed):
    """Symmetric diagonally dominant matrix with power-law row lengths (a
    few long rows among many short ones): where sorting rows by length in
    SELL-C-sigma removes padding."""
    rng = np.random.default_rng(seed)
    deg = np.minimum((rng.pareto(1.5, n) * 3).astype(int) + 1, 200)
    rows, cols = [], []
    for i in range(n):
        c = rng.choice(n, size=min(deg[i], n), replace=False)
        rows.append(np.full(c.shape[0], i))
        cols.append(c)
    r = np.concatenate(rows)
    c = np.concatenate(cols)
    import scipy.sparse as sp
    A = sp.coo_matrix((rng.standard_normal(r.shape[0]), (r, c)), shape=(n, n)).tocsr()
    A = A + A.T
    A = A + sp.diags(np.asarray(abs(A).sum(axis=1)).ravel() + 1.0)
    A = A.tocsr()
    A.sort_indices()
    return P.CSRSystem(0, 0, A.indptr.astype(np.int32), A.indices.astype(np.int32), A.data.astype(np.float64),
                       rng.random(n), np.zeros(n, bool), f"ragged_{n}")


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_sell_c_sigma_gives_the_sell32_bits(plat, dtype):
    """SELL-C-sigma (C = 8/16/32 rows per slice, rows sorted by length within
    windows of sigma rows, widths 1/2/4, int32 or int16 columns) adds each
    row's products in stored order like SELL-32, so every variant gives its
    bits; on the ragged matrix sorting cuts the padding."""
    cases = [P.poisson_2d(100), P.q1_system(3, 10, 3, 2.0), P.random_spd(257, 3, density=0.02, empty_rows=5),
             P.random_spd(33, 2, empty_rows=3), _ragged(3000, 5)]
    for s in cases:
        xs = P.uniform01(8, s.n, stream=9) - 0.5
        A = _mat(plat, s, dtype)
        A.set_format(FMT_SELL, 1)
        x = _vec(plat, xs, dtype)
        y0 = x.CloneWithoutContent()
        A.VectorMult(x, y0)
        ref = y0.numpy()
        for col16 in (False, True):
            for C in (8, 16, 32):
                for sigma in (1, 64, 1024):
                    for w in (1, 2, 4):
                        try:
                            A.set_sell(C, sigma, w, col16)
                        except B200LAError as e:
                            assert col16 and e.status == -7  # far columns: int16 offsets refused
                            continue
                        assert A.get_sell() == (C, sigma if sigma == 1 else -(-sigma // C) * C)
                        y = x.CloneWithoutContent()
                        A.VectorMult(x, y)
                        np.testing.assert_array_equal(y.numpy(), ref, err_msg=f"{s.name} C{C} s{sigma} w{w} {col16}")
                        # y += A x through the same schedule
                        A.VectorMultAdd(x, y)
                        np.testing.assert_array_equal(y.numpy(), (ref + ref).astype(ref.dtype))


def test_sell_c_sigma_in_the_solver_and_the_tuner(plat):
    s = _ragged(4000, 7)
    A = _mat(plat, s)
    A.set_sell(16, 512, 2, False)
    b = _vec(plat, s.b)
    x = _vec(plat, np.zeros(s.n))
    cg = lmp.setup_CG_solver(maxits=5000, atol=0.0, rtol=1e-10, dtol=1e8)
    cg.SetupOperator(A)
    assert cg.Solve(b, x) == lmp.kSolverSuccess
    ref = oracle.cg(s.rowptr, s.col, s.val, s.b, maxits=5000, atol=0.0, rtol=1e-10)
    assert abs(cg.iter() - ref.iters) <= 1
    assert np.linalg.norm(x.numpy() - ref.x) <= 1e-10 * np.linalg.norm(ref.x)
    # the schedule changes under the solver: its graph is captured again
    A.set_sell(8, 1, 1, False)
    x2 = _vec(plat, np.zeros(s.n))
    assert cg.Solve(b, x2) == lmp.kSolverSuccess
    assert np.linalg.norm(x2.numpy() - ref.x) <= 1e-10 * np.linalg.norm(ref.x)
    fmt, prm, us = A.tune()
    assert us > 0 and fmt in (FMT_CSR, FMT_SELL, FMT_SELL16)  # no stencil on the ragged matrix
    if fmt != FMT_CSR:
        C, sigma = A.get_sell()
        assert C in (8, 16, 32) and sigma in (1, 1024)


def _off_stencil(s):
    """The system with one extra entry in a short (border) row at an offset no
    row of the matrix has: the longest rows keep the stencil, this row leaves
    it."""
    lens = np.diff(s.rowptr)
    r = int(np.flatnonzero(lens < lens.max())[0])
    lo, hi = int(s.rowptr[r]), int(s.rowptr[r + 1])
    cols = s.col[lo:hi]
    c = r + int(np.abs(s.col - np.repeat(np.arange(s.n), lens)).max()) + 1
    c = c if c < s.n else r - (c - r)
    pos = lo + int(np.searchsorted(cols, c))
    col = np.insert(s.col, pos, c).astype(np.int32)
    val = np.insert(s.val, pos, 0.25)
    rowptr = s.rowptr.copy()
    rowptr[r + 1:] += 1
    return P.CSRSystem(s.dim, s.cells, rowptr, col, val, s.b, s.boundary, s.name + "_off")


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_stencil_copy_gives_the_sell_bits(plat, dtype):
    """The values-only copy (B200LA_FMT_STENCIL: no column storage, entry k
    of a row at column row + stencil[k]) adds each row's products in its
    stored (ascending column) order, so y = A x and y += A x are SELL's bits
    for every width, on 2D (9-entry) and 3D (27-entry) Q1 matrices with
    Dirichlet rows and a ragged last slice; matrices without a 9/27-entry
    stencil are refused with B200LA_ERR_UNSUPPORTED."""
    cases = [P.poisson_2d(40), P.q1_system(2, 37, 5, 1.0), P.q1_system(3, 11, 3, 2.0), P.q1_system(3, 6, 4, 0.5)]
    for s in cases:
        xs = P.uniform01(8, s.n, stream=9) - 0.5
        A = _mat(plat, s, dtype)
        A.set_format(FMT_SELL, 1)
        x = _vec(plat, xs, dtype)
        y0 = x.CloneWithoutContent()
        A.VectorMult(x, y0)
        ref = y0.numpy()
        E = int(np.diff(s.rowptr).max())
        for w in (1, 2, 4):
            A.set_format(FMT_STENCIL, w)
            assert A.get_format() == (FMT_STENCIL, w)
            assert A.sell_padded() == -(-s.n // 32) * 32 * (-(-E // w) * w)
            y = x.CloneWithoutContent()
            A.VectorMult(x, y)
            np.testing.assert_array_equal(y.numpy(), ref, err_msg=f"{s.name} w{w}")
            A.VectorMultAdd(x, y)
            np.testing.assert_array_equal(y.numpy(), (ref + ref).astype(ref.dtype))
    for bad in (P.random_spd(300, 3, density=0.02, empty_rows=5), _ragged(2000, 5), _off_stencil(P.poisson_2d(20)),
                _off_stencil(P.q1_system(3, 5, 1, 1.0))):
        A = _mat(plat, bad, dtype)
        with pytest.raises(B200LAError) as e:
            A.set_format(FMT_STENCIL, 1)
        assert e.value.status == -7, bad.name
        # the matrix still works on its previous schedule
        x = _vec(plat, np.ones(bad.n), dtype)
        y = x.CloneWithoutContent()
        A.VectorMult(x, y)
        np.testing.assert_allclose(y.numpy(), oracle.spmv(bad.rowptr, bad.col, bad.val, np.ones(bad.n)),
                                   rtol=1e-5 if dtype == np.float32 else 1e-13, atol=1e-6)


def test_stencil_copy_in_the_solvers(plat):
    """CG on the values-only copy takes the SELL16 path's iterations and
    solution bits (3D Q1, FP64, Jacobi); ZeroRows rebuilds the copy with the
    new values; the tuner may pick it on a Q1 matrix and CG then matches the
    oracle."""
    s = P.q1_system(3, 14, 11, 1.0)
    b = _vec(plat, s.b)
    out = []
    for fmt, w in ((FMT_SELL16, 1), (FMT_STENCIL, 1), (FMT_STENCIL, 4)):
        A = _mat(plat, s)
        A.set_format(fmt, w)
        x = _vec(plat, np.zeros(s.n))
        solver = lmp.setup_CG_solver(maxits=5000, atol=0.0, rtol=1e-10, dtol=1e8)
        solver.SetupOperator(A)
        assert solver.Solve(b, x) == lmp.kSolverSuccess
        out.append((solver.iter(), x.numpy()))
    for it, xs in out[1:]:
        assert it == out[0][0]
        np.testing.assert_array_equal(xs, out[0][1])
    ref = oracle.cg(s.rowptr, s.col, s.val, s.b, maxits=5000, atol=0.0, rtol=1e-10, precond=True)
    assert abs(out[0][0] - ref.iters) <= 1
    # ZeroRows on the values-only schedule: the copy follows the new values
    rows = np.arange(5, s.n, 97, dtype=np.int32)
    A1, A2 = _mat(plat, s), _mat(plat, s)
    A1.set_format(FMT_SELL, 1)
    A2.set_format(FMT_STENCIL, 2)
    for A in (A1, A2):
        A.ZeroRows(rows, 3.0)
    assert A2.get_format() == (FMT_STENCIL, 2)
    xv = _vec(plat, P.uniform01(2, s.n, stream=3))
    y1, y2 = xv.CloneWithoutContent(), xv.CloneWithoutContent()
    A1.VectorMult(xv, y1)
    A2.VectorMult(xv, y2)
    np.testing.assert_array_equal(y1.numpy(), y2.numpy())
    # CastTo keeps the schedule: the FP32 copy is values-only too, with the
    # FP32 SELL copy's bits
    A3 = A2.CastTo(np.float32)
    assert A3.get_format() == (FMT_STENCIL, 2) and A3.get_sell() == (32, 1)
    x32 = _vec(plat, P.uniform01(4, s.n, stream=5), np.float32)
    y3, y4 = x32.CloneWithoutContent(), x32.CloneWithoutContent()
    A3.VectorMult(x32, y3)
    A3.set_format(FMT_SELL, 1)
    A3.VectorMult(x32, y4)
    np.testing.assert_array_equal(y3.numpy(), y4.numpy())
    # the tuner on a Q1 matrix keeps one of the schedules it timed
    A = _mat(plat, P.q1_system(2, 120, 2, 1.0))
    fmt, prm, us = A.tune()
    assert fmt in (FMT_CSR, FMT_SELL, FMT_SELL16, FMT_STENCIL) and us > 0

