"""The CPU oracle, pinned against the reference's own known answers and runs.

Mirrors tests/cg_test.cc, tests/lmp_test.cc and tests/cuda_test.cc of the
reference (3x3 known answers, tolerance 1e-12), then checks the C restatement
bit for bit against runs of the reference's compiled lmp sources recorded in
tests/golden/ (make_golden.py).
"""
import hashlib
import json
import os

import numpy as np
import pytest

import oracle
from ba_b200 import problems as P

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def _golden_cases():
    with open(os.path.join(GOLD, "reference_cg_runs.json")) as f:
        return json.load(f)["cases"]


def _system(name):
    import re
    m = re.match(r"poisson2d_(\d+)$", name)
    if m:
        return P.poisson_2d(int(m.group(1)))
    table = {
        "varcoef2d_33_s1": lambda: P.q1_system(2, 33, 11, 1.0, "varcoef2d_33_s1"),
        "poisson3d_8": lambda: P.q1_system(3, 8, 12, 0.0, "poisson3d_8"),
        "varcoef3d_12_s2": lambda: P.q1_system(3, 12, 13, 2.0, "varcoef3d_12_s2"),
        "random_spd_17": lambda: P.random_spd(17, 1, empty_rows=0),
        "random_spd_33": lambda: P.random_spd(33, 2, empty_rows=3),
        "random_spd_257": lambda: P.random_spd(257, 3, density=0.02, empty_rows=5),
    }
    return table[name]()


def test_cg_test_known_answer():
    # tests/cg_test.cc:44-94: cg() with rel_eps = abs_eps = 0, max_iter 100
    kat = json.load(open(os.path.join(GOLD, "reference_known_answers.json")))
    s = P.known_answer_3x3()
    r = oracle.lmp_cg(s.rowptr, s.col, s.val, s.b, rel_eps=0.0, abs_eps=0.0, max_iter=100)
    np.testing.assert_allclose(r.x, kat["cg_test_3x3"]["x"], rtol=0, atol=1e-12)
    for precond in (False, True):
        r = oracle.cg(s.rowptr, s.col, s.val, s.b, maxits=100, atol=0.0, rtol=1e-14,
                      precond=precond)
        np.testing.assert_allclose(r.x, kat["cg_test_3x3"]["x"], rtol=0, atol=1e-12)


def test_lmp_and_cuda_spmv_known_answers():
    kat = json.load(open(os.path.join(GOLD, "reference_known_answers.json")))
    s7 = P.lmp_test_3x3()
    y = oracle.spmv(s7.rowptr, s7.col, s7.val, kat["lmp_test_spmv"]["x"])
    np.testing.assert_array_equal(y, kat["lmp_test_spmv"]["y"])
    s9 = P.known_answer_3x3()
    y = oracle.spmv(s9.rowptr, s9.col, s9.val, kat["cuda_test_spmv"]["x"])
    np.testing.assert_allclose(y, kat["cuda_test_spmv"]["y"], rtol=0, atol=1e-12)


@pytest.mark.parametrize("case", _golden_cases(), ids=lambda c: c["name"])
def test_oracle_matches_reference_runs(case):
    s = _system(case["name"])
    assert s.n == case["n"] and s.nnz == case["nnz"]
    assert _sha(s.rowptr) == case["sha_rowptr"] and _sha(s.col) == case["sha_col"]
    assert _sha(s.val) == case["sha_val"] and _sha(s.b) == case["sha_b"]
    for run in case["runs"]:
        dt = np.float64 if run["dtype"] == "f64" else np.float32
        r = oracle.cg(s.rowptr, s.col, s.val, s.b, maxits=20000, atol=0.0, rtol=run["rtol"],
                      dtol=1e8, precond=run["precond"], dtype=dt)
        assert r.iters == run["iters"]
        assert r.state == run["state"]
        assert r.res == run["res"] and r.res_init == run["res_init"]
        assert _sha(r.x) == run["sha_x"]          # bit-identical to the reference
    lr = oracle.lmp_cg(s.rowptr, s.col, s.val, s.b, rel_eps=1e-10, abs_eps=0.0, max_iter=20000)
    assert lr.iters == case["lmp_cg"]["max_iter_out"]
    assert _sha(lr.x) == case["lmp_cg"]["sha_x"]
    xs = P.uniform01(case["spmv"]["x_seed"], s.n, stream=case["spmv"]["x_stream"])
    y = oracle.spmv(s.rowptr, s.col, s.val, xs)
    if "y" in case["spmv"]:
        np.testing.assert_array_equal(y, case["spmv"]["y"])
    else:
        assert _sha(y) == case["spmv"]["sha_y"]


@pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built")
def test_oracle_matches_compiled_reference_live():
    s = P.q1_system(2, 48, 5, 1.5, "live")
    for dt, rtol in ((np.float64, 1e-10), (np.float32, 1e-5)):
        a = oracle.cg(s.rowptr, s.col, s.val, s.b, maxits=5000, atol=0.0, rtol=rtol, dtype=dt)
        b = oracle.ref_cg(s.rowptr, s.col, s.val, s.b, maxits=5000, atol=0.0, rtol=rtol, dtype=dt)
        assert a.iters == b.iters and np.array_equal(a.x, b.x)
    y1 = oracle.spmv(s.rowptr, s.col, s.val, s.b)
    y2 = oracle.ref_spmv(s.rowptr, s.col, s.val, s.b, impl=oracle.IMPL_OPENMP, nthreads=2)
    np.testing.assert_array_equal(y1, y2)


def test_iterate_control_semantics():
    # common/iterate_control.cc:80-107
    chk = oracle.iterate_check
    st, first = chk(0, 10.0, 100, 1e-12, 1e-8, 1e8, 0.0)
    assert st == oracle.CTRL_ITERATE and first == 10.0
    assert chk(5, 1e-13, 100, 1e-12, 1e-8, 1e8, first)[0] == oracle.CTRL_SUCCESS_ABS
    assert chk(5, 1e-12, 100, 1e-12, 1e-8, 1e8, first)[0] == oracle.CTRL_SUCCESS_ABS  # <=
    assert chk(5, 1e-7, 100, 0.0, 1e-8, 1e8, first)[0] == oracle.CTRL_ITERATE     # strict <
    assert chk(5, 9.9e-8, 100, 0.0, 1e-8, 1e8, first)[0] == oracle.CTRL_SUCCESS_REL
    assert chk(5, 1e10, 100, 0.0, 1e-8, 1e8, first)[0] == oracle.CTRL_FAIL_DIV
    assert chk(100, 1.0, 100, 0.0, 1e-8, 1e8, first)[0] == oracle.CTRL_FAIL_MAXITS


def test_maxits_and_zero_rhs():
    s = P.poisson_2d(16)
    r = oracle.cg(s.rowptr, s.col, s.val, s.b, maxits=7, atol=0.0, rtol=1e-10)
    assert r.iters == 7 and r.state == oracle.CTRL_FAIL_MAXITS
    r = oracle.cg(s.rowptr, s.col, s.val, np.zeros(s.n), maxits=7, atol=0.0, rtol=1e-10)
    assert r.iters == 0 and r.state == oracle.CTRL_SUCCESS_ABS and not r.x.any()


def test_mpir_reaches_fp64_solution():
    s = P.q1_system(2, 40, 3, 1.0, "mp")
    ref = oracle.cg(s.rowptr, s.col, s.val, s.b, maxits=10000, atol=0.0, rtol=1e-12)
    mp, outer = oracle.mpir(s.rowptr, s.col, s.val, s.b, rtol=1e-10, inner_rtol=1e-4)
    assert mp.state == 0 and outer >= 2
    assert mp.res <= 1e-10 * mp.res_init
    assert np.linalg.norm(mp.x - ref.x) <= 1e-8 * np.linalg.norm(ref.x)


def test_generator_shapes():
    # 2D Poisson, 256^2 cells -> 66,049 DOFs, 591,361 nnz; Q1 counts (3n+1)^d nnz
    c1 = P.poisson_2d(256)
    assert c1.n == 66049 and c1.nnz == 591361
    for n in (4, 9, 13):
        s = P.poisson_3d(n)
        assert s.n == (n + 1) ** 3 and s.nnz == (3 * n + 1) ** 3
        assert np.all(np.diff(s.col[s.rowptr[0]:s.rowptr[1]]) > 0)
    s = P.poisson_3d(6)
    # interior row: centre 8h/3, 12 edge -h/6, 8 corner -h/12, 6 faces stored 0
    i = 3 + 7 * (3 + 7 * 3)
    row = s.val[s.rowptr[i]:s.rowptr[i + 1]]
    h = 1.0 / 6
    assert row.shape[0] == 27
    assert np.isclose(row[13], 8 * h / 3) and np.sum(row == 0.0) == 6
    assert np.isclose(row.sum(), 0.0, atol=1e-15)
    # Dirichlet row: full pattern, identity values
    assert s.boundary[0] and s.val[s.rowptr[0]] == 1.0
    assert np.all(s.val[s.rowptr[0] + 1:s.rowptr[1]] == 0.0)
    assert np.all(s.b[s.boundary] == 0.0)
    sizes = P.batch_sizes(1024)
    assert sizes.min() >= 16 and sizes.max() <= 256


# ---- Jacobi<LAD>, BiCGSTAB<LAD> and GMRES<LAD> -----------------------------------

def _krylov_cases():
    with open(os.path.join(GOLD, "reference_krylov_runs.json")) as f:
        return json.load(f)["cases"]


def _krylov_system(name):
    import re
    m = re.match(r"convdiff2d_(\d+)_pe([0-9.]+)$", name)
    if m:
        return P.convdiff_2d(int(m.group(1)), float(m.group(2)))
    return _system(name)


@pytest.mark.parametrize("case", _krylov_cases(), ids=lambda c: c["name"])
def test_jacobi_bicgstab_gmres_oracle_matches_reference_runs(case):
    s = _krylov_system(case["name"])
    assert s.n == case["n"] and s.nnz == case["nnz"]
    assert _sha(s.val) == case["sha_val"] and _sha(s.b) == case["sha_b"]
    for run in case["jacobi"]:
        r = oracle.jacobi(s.rowptr, s.col, s.val, s.b, mode=run["mode"], maxits=run["maxits"],
                          inner_iter=run["inner_iter"], smooth_iter=run["smooth_iter"], w=run["w"],
                          atol=0.0, rtol=run["rtol"], dtol=1e8)
        assert (r.iters, r.state) == (run["iters"], run["state"])
        assert r.res == run["res"] and r.res_init == run["res_init"]
        assert _sha(r.x) == run["sha_x"]          # bit-identical to the reference
    for run in case["bicgstab"]:
        r, restarts = oracle.bicgstab(s.rowptr, s.col, s.val, s.b, maxits=run["maxits"], atol=0.0,
                                      rtol=run["rtol"], dtol=1e8, precond=run["precond"])
        assert (r.iters, r.state, restarts) == (run["iters"], run["state"], run["restarts"])
        assert r.res == run["res"]
        assert _sha(r.x) == run["sha_x"]
    for run in case["gmres"]:
        r = oracle.gmres(s.rowptr, s.col, s.val, s.b, size_basis=run["size_basis"], maxits=run["maxits"],
                         atol=0.0, rtol=run["rtol"], dtol=1e8, precond=run["precond"])
        assert (r.iters, r.state) == (run["iters"], run["state"])
        assert r.res == run["res"] and r.res_init == run["res_init"]
        assert _sha(r.x) == run["sha_x"]


def test_jacobi_bicgstab_gmres_known_answer():
    # the 3x3 system of tests/cg_test.cc:44-94 (x = (-0.25, -1.5, -0.75))
    kat = json.load(open(os.path.join(GOLD, "reference_known_answers.json")))
    s = P.known_answer_3x3()
    for precond in (False, True):
        r, _ = oracle.bicgstab(s.rowptr, s.col, s.val, s.b, maxits=100, atol=0.0, rtol=1e-15,
                               precond=precond)
        np.testing.assert_allclose(r.x, kat["cg_test_3x3"]["x"], rtol=0, atol=1e-12)
    r = oracle.jacobi(s.rowptr, s.col, s.val, s.b, maxits=5000, atol=0.0, rtol=1e-15)
    np.testing.assert_allclose(r.x, kat["cg_test_3x3"]["x"], rtol=0, atol=1e-12)
    for precond in (False, True):
        r = oracle.gmres(s.rowptr, s.col, s.val, s.b, size_basis=3, maxits=100, atol=0.0, rtol=1e-15,
                         precond=precond)
        np.testing.assert_allclose(r.x, kat["cg_test_3x3"]["x"], rtol=0, atol=1e-12)


def indefinite_2x2():
    return (np.array([0, 1, 2], np.int32), np.array([0, 1], np.int32), np.array([1.0, -1.0]),
            np.array([1.0, 1.0]))


def test_bicgstab_restart_and_short_update():
    rp, c, v, b = indefinite_2x2()
    # no preconditioner: sigma = (A r0).r0 = 0 at every step, so each step
    # restarts (bicgstab.h:282-284) until IterateControl stops at maxits
    r, restarts = oracle.bicgstab(rp, c, v, b, maxits=5, atol=0.0, rtol=1e-12, precond=False)
    assert (r.iters, r.state, restarts) == (5, oracle.CTRL_FAIL_MAXITS, 5)
    # Jacobi: q = (1, -1), A q = (1, 1), alpha = 1, s = 0 -> the short update
    # lands on the exact solution (1, -1)
    r, restarts = oracle.bicgstab(rp, c, v, b, maxits=5, atol=0.0, rtol=1e-12, precond=True)
    assert (r.iters, r.state, restarts) == (1, oracle.CTRL_SUCCESS_ABS, 0)
    np.testing.assert_array_equal(r.x, [1.0, -1.0])
    if oracle.ref_available():
        for pc in (False, True):
            a, ra = oracle.bicgstab(rp, c, v, b, maxits=5, atol=0.0, rtol=1e-12, precond=pc)
            e, re_ = oracle.ref_bicgstab(rp, c, v, b, maxits=5, atol=0.0, rtol=1e-12, precond=pc)
            assert (a.iters, a.state, ra) == (e.iters, e.state, re_) and np.array_equal(a.x, e.x)


@pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built")
def test_jacobi_bicgstab_gmres_match_compiled_reference_live():
    s = P.convdiff_2d(20, 50.0)
    for mode, w in ((0, 1.0), (1, 0.8), (2, 1.0), (3, 0.5)):
        kw = dict(mode=mode, maxits=50 if mode == 3 else 4000, inner_iter=2, smooth_iter=3, w=w,
                  atol=0.0, rtol=1e-7, dtol=1e8)
        a = oracle.jacobi(s.rowptr, s.col, s.val, s.b, **kw)
        e = oracle.ref_jacobi(s.rowptr, s.col, s.val, s.b, **kw)
        assert (a.iters, a.state) == (e.iters, e.state) and np.array_equal(a.x, e.x)
    for pc in (False, True):
        a, ra = oracle.bicgstab(s.rowptr, s.col, s.val, s.b, maxits=500, atol=0.0, rtol=1e-11, precond=pc)
        e, re_ = oracle.ref_bicgstab(s.rowptr, s.col, s.val, s.b, maxits=500, atol=0.0, rtol=1e-11,
                                     precond=pc)
        assert (a.iters, ra) == (e.iters, re_) and np.array_equal(a.x, e.x)
    for pc in (False, True):
        for m in (7, 40):
            a = oracle.gmres(s.rowptr, s.col, s.val, s.b, size_basis=m, maxits=800, atol=0.0, rtol=1e-11,
                             precond=pc)
            e = oracle.ref_gmres(s.rowptr, s.col, s.val, s.b, size_basis=m, maxits=800, atol=0.0, rtol=1e-11,
                                 precond=pc)
            assert (a.iters, a.state) == (e.iters, e.state) and np.array_equal(a.x, e.x)


# ---- TransformFromCOO -----------------------------------------------------------

LMP_TEST_COO = ([0, 0, 1, 1, 1, 2, 2], [0, 1, 0, 1, 2, 1, 2], [2.0, -1.0, -1.0, 2.0, -1.0, -1.0, 2.0])


def test_coo_to_csr_known_answer():
    # tests/lmp_test.cc:42-89: the 7 triplets through TransformFromCOO, then
    # A (1, -2, 0) = (4, -5, 2); here also in reversed order
    kat = json.load(open(os.path.join(GOLD, "reference_known_answers.json")))
    s7 = P.lmp_test_3x3()
    for order in (slice(None), slice(None, None, -1)):
        rows, cols, vals = (np.asarray(a)[order] for a in LMP_TEST_COO)
        rp, c, v = oracle.coo_to_csr(3, 3, rows, cols, vals)
        np.testing.assert_array_equal(rp, s7.rowptr)
        np.testing.assert_array_equal(c, s7.col)
        np.testing.assert_array_equal(v, s7.val)
        np.testing.assert_array_equal(oracle.spmv(rp, c, v, kat["lmp_test_spmv"]["x"]), kat["lmp_test_spmv"]["y"])


def test_coo_to_csr_matches_reference_runs():
    from tests.golden.make_golden import coo_triplets
    with open(os.path.join(GOLD, "reference_krylov_runs.json")) as f:
        cases = json.load(f)["coo_to_csr"]
    for case in cases:
        rows, cols, vals = coo_triplets(case["nrow"], case["ncol"], case["nnz"], case["seed"])
        rp, c, v = oracle.coo_to_csr(case["nrow"], case["ncol"], rows, cols, vals)
        assert (_sha(rp), _sha(c), _sha(v)) == (case["sha_rowptr"], case["sha_col"], case["sha_val"])
    with pytest.raises(ValueError):
        oracle.coo_to_csr(3, 3, [0, 3], [0, 0], [1.0, 1.0])


def test_kept_direction_refinement_restatement():
    # the device's default fused refinement restated: FP32 PCG whose residual
    # is replaced by the FP64 one every 10x reduction, direction kept.  It
    # reaches the FP64 tolerance in fewer inner iterations than restarting the
    # inner solve every pass (MPIR's form), close to the FP64 PCG's count
    for dim, n, sigma in ((2, 48, 1.0), (3, 20, 2.0)):
        s = P.q1_system(dim, n, 77 + n, sigma)
        kept, passes = oracle.mpcg_kept(s.rowptr, s.col, s.val, s.b, rtol=1e-10, inner_rtol=0.1)
        rst, _ = oracle.mpir(s.rowptr, s.col, s.val, s.b, rtol=1e-10, inner_rtol=1e-5)
        f64 = oracle.cg(s.rowptr, s.col, s.val, s.b, maxits=100000, atol=0.0, rtol=1e-10)
        assert kept.state == 0 and passes >= 5
        r = s.b - oracle.spmv(s.rowptr, s.col, s.val, kept.x)
        assert np.linalg.norm(r) < 1e-10 * np.linalg.norm(s.b)
        assert kept.iters < rst.iters and kept.iters <= 1.3 * f64.iters, (kept.iters, rst.iters, f64.iters)
