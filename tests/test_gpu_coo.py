"""COO -> CSR on the device (CPU_CSR_lMatrix::TransformFromCOO,
lmp/lmatrix_csr_cpu.cc:883-906) against the CPU oracle, which is pinned bit for
bit to the reference's own TransformFromCOO in tests/test_oracle.py.

Bar: the device CSR (row pointer, column order, values) equals the oracle's
bit for bit, duplicates and empty rows included, from host arrays and from
device buffers; the reference's lmp_test known answer holds; bad triplets are
refused.
"""
import json
import os

import numpy as np
import pytest

import oracle
from ba_b200 import lmp
from ba_b200 import problems as P
from ba_b200._lib import B200LAError

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
LMP_TEST_COO = ([0, 0, 1, 1, 1, 2, 2], [0, 1, 0, 1, 2, 1, 2], [2.0, -1.0, -1.0, 2.0, -1.0, -1.0, 2.0])


@pytest.fixture(scope="module")
def plat():
    return lmp.init_platform(0)


def _triplets(nrow, ncol, nnz, seed):
    rng = np.random.default_rng(seed)
    return (rng.integers(0, nrow, nnz).astype(np.int32), rng.integers(0, ncol, nnz).astype(np.int32),
            rng.standard_normal(nnz))


def test_lmp_test_known_answer(plat):
    kat = json.load(open(os.path.join(GOLD, "reference_known_answers.json")))
    s7 = P.lmp_test_3x3()
    for order in (slice(None), slice(None, None, -1)):
        rows, cols, vals = (np.asarray(a)[order] for a in LMP_TEST_COO)
        A = lmp.B200_CSR_lMatrix.TransformFromCOO(rows, cols, vals, 3, 3, platform=plat)
        rp, c, v = A.csr()
        np.testing.assert_array_equal(rp, s7.rowptr)
        np.testing.assert_array_equal(c, s7.col)
        np.testing.assert_array_equal(v, s7.val)
        x = lmp.B200_lVector.from_numpy(kat["lmp_test_spmv"]["x"], platform=plat)
        y = x.CloneWithoutContent()
        A.VectorMult(x, y)
        np.testing.assert_array_equal(y.numpy(), kat["lmp_test_spmv"]["y"])


@pytest.mark.parametrize("nrow,ncol,nnz,seed", [(50, 60, 400, 1), (300, 300, 5000, 2), (1000, 800, 3000, 3),
                                                (20000, 20000, 400000, 4), (7, 7, 0, 5)])
def test_random_triplets_match_oracle(plat, nrow, ncol, nnz, seed):
    rows, cols, vals = _triplets(nrow, ncol, nnz, seed)
    ref = oracle.coo_to_csr(nrow, ncol, rows, cols, vals)
    A = lmp.B200_CSR_lMatrix.TransformFromCOO(rows, cols, vals, nrow, ncol, platform=plat)
    for got, want in zip(A.csr(), ref):
        np.testing.assert_array_equal(got, want)
    A32 = lmp.B200_CSR_lMatrix.TransformFromCOO(rows, cols, vals, nrow, ncol, platform=plat, dtype=np.float32)
    rp, c, v = A32.csr()
    np.testing.assert_array_equal(rp, ref[0])
    np.testing.assert_array_equal(c, ref[1])
    np.testing.assert_array_equal(v, ref[2].astype(np.float32))


def test_float32_values_into_both_storage_types(plat):
    # float32 triplet values: cast to FP64 storage exactly, kept as FP32
    rows, cols, vals = _triplets(400, 300, 6000, 7)
    v32 = vals.astype(np.float32)
    ref = oracle.coo_to_csr(400, 300, rows, cols, v32.astype(np.float64))
    for dt in (np.float64, np.float32):
        A = lmp.B200_CSR_lMatrix.TransformFromCOO(rows, cols, v32, 400, 300, platform=plat, dtype=dt)
        rp, c, v = A.csr()
        np.testing.assert_array_equal(rp, ref[0])
        np.testing.assert_array_equal(c, ref[1])
        np.testing.assert_array_equal(v, ref[2].astype(dt))


def test_long_and_distinct_rows(plat):
    # the warp-per-row kernel ranks distinct columns with shuffles for rows
    # of up to 256 entries and falls back to the selection sort for longer
    # rows or repeated columns; cover each side of both limits
    rng = np.random.default_rng(11)
    lengths = [0, 1, 31, 32, 33, 64, 100, 255, 256, 257, 600, 27, 125]
    ncol = 1000
    rows, cols = [], []
    for r, L in enumerate(lengths):
        rows.append(np.full(L, r, np.int32))
        cols.append(rng.permutation(ncol)[:L].astype(np.int32))   # distinct columns
    # two rows with one repeated column each (short and long)
    for L in (40, 300):
        r = len(lengths)
        lengths.append(L)
        cc = rng.permutation(ncol)[:L].astype(np.int32)
        cc[L // 2] = cc[3]
        rows.append(np.full(L, r, np.int32))
        cols.append(cc)
    rows, cols = np.concatenate(rows), np.concatenate(cols)
    perm = rng.permutation(rows.size)
    rows, cols = rows[perm], cols[perm]
    vals = rng.standard_normal(rows.size)
    nrow = len(lengths)
    ref = oracle.coo_to_csr(nrow, ncol, rows, cols, vals)
    A = lmp.B200_CSR_lMatrix.TransformFromCOO(rows, cols, vals, nrow, ncol, platform=plat)
    for got, want in zip(A.csr(), ref):
        np.testing.assert_array_equal(got, want)


def test_device_triplets_and_scrambled_fe_matrix(plat):
    import torch
    s = P.q1_system(3, 40, 21, 1.0, "q1_40")
    rows = np.repeat(np.arange(s.n, dtype=np.int32), np.diff(s.rowptr))
    perm = np.random.default_rng(9).permutation(s.nnz)
    r, c, v = rows[perm], s.col[perm], s.val[perm]
    dev = [torch.from_numpy(a).cuda() for a in (r, c, v)]
    for src in ((r, c, v), tuple(dev)):
        A = lmp.B200_CSR_lMatrix.TransformFromCOO(*src, s.n, s.n, platform=plat)
        rp, cc, vv = A.csr()
        # no duplicates: the sorted rows are the generator's CSR exactly
        np.testing.assert_array_equal(rp, s.rowptr)
        np.testing.assert_array_equal(cc, s.col)
        np.testing.assert_array_equal(vv, s.val)
    # the built matrix solves like the uploaded one (same diagonal positions)
    b = lmp.B200_lVector.from_numpy(s.b, platform=plat)
    x = lmp.B200_lVector.from_numpy(np.zeros(s.n), platform=plat)
    solver = lmp.setup_CG_solver(maxits=5000, atol=0.0, rtol=1e-10, dtol=1e8)
    solver.SetupOperator(A)
    assert solver.Solve(b, x) == lmp.kSolverSuccess
    ref = oracle.cg(s.rowptr, s.col, s.val, s.b, maxits=5000, atol=0.0, rtol=1e-10)
    assert abs(solver.iter() - ref.iters) <= 1


def test_csr_download_into_given_buffers(plat):
    import torch
    rows, cols, vals = _triplets(300, 300, 5000, 2)
    ref = oracle.coo_to_csr(300, 300, rows, cols, vals)
    pin = [torch.from_numpy(a).pin_memory().numpy() for a in (rows, cols, vals)]
    A = lmp.B200_CSR_lMatrix.TransformFromCOO(*pin, 300, 300, platform=plat)
    out = (np.empty(301, np.int32), torch.empty(5000, dtype=torch.int32, pin_memory=True).numpy(),
           np.empty(5000, np.float64))
    got = A.csr(out=out)
    for g, o, w in zip(got, out, ref):
        assert np.shares_memory(g, o)
        np.testing.assert_array_equal(g, w)
    with pytest.raises(B200LAError):
        A.csr(out=(np.empty(301, np.int32), np.empty(4999, np.int32), np.empty(5000, np.float64)))
    with pytest.raises(B200LAError):
        A.csr(out=(np.empty(301, np.int32), np.empty(5000, np.int32), np.empty(5000, np.float32)))


def test_bad_triplets_are_refused(plat):
    with pytest.raises(B200LAError):
        lmp.B200_CSR_lMatrix.TransformFromCOO([0, 3], [0, 0], [1.0, 1.0], 3, 3, platform=plat)
    with pytest.raises(B200LAError):
        lmp.B200_CSR_lMatrix.TransformFromCOO([0, 1], [0, -1], [1.0, 1.0], 3, 3, platform=plat)
    # the context stays usable
    A = lmp.B200_CSR_lMatrix.TransformFromCOO(*LMP_TEST_COO, 3, 3, platform=plat)
    assert A.get_nnz() == 7
