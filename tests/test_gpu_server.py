"""The request loop on the GPU: a Poisson-arrival stream of host-CSR and
device-assembled solves, admission by the HBM budget, isolation (each result
bit for bit the same alone and in the mix), and host-side fault injection
(malformed, oversized and non-finite requests fail alone; the server keeps
serving the rest)."""
import time

import numpy as np
import pytest

import oracle
from ba_b200 import lmp
from ba_b200 import problems as P
from ba_b200.batch import slot_bytes
from ba_b200.server import Server

pytestmark = pytest.mark.gpu

RTOL = 1e-8


@pytest.fixture(scope="module")
def plat():
    return lmp.init_platform(0)


def _true_rel_res(s, x):
    return np.linalg.norm(s.b - oracle.spmv(s.rowptr, s.col, s.val, x)) / np.linalg.norm(s.b)


def _stream(count=36, rate=400.0):
    """Small requests: DOFs log-uniform in [1e2, 2e4], 2D and 3D, sigma in
    [0.5, 2]; a third of them arrive as host CSR, the rest are assembled on
    the device."""
    return P.serve_stream(count, rate=rate, lo_dofs=1e2, hi_dofs=2e4, seed=P.SEED_SERVE + 7)


def _submit(S, req, k):
    if k % 3 == 0:
        s = P.q1_system(req["dim"], req["cells"], req["seed"], req["sigma"])
        return S.submit_system(s), s
    return S.submit_q1(req["dim"], req["cells"], req["seed"], req["sigma"]), None


def test_stream_isolation_and_tolerance(plat):
    reqs = _stream()
    got = {}
    with Server(16, rtol=RTOL, platform=plat) as S:
        t0 = time.monotonic()
        ids = []
        for k, rq in enumerate(reqs):
            delay = t0 + rq["t"] - time.monotonic()
            if delay > 0:
                time.sleep(delay)
            ids.append(_submit(S, rq, k))
        S.drain(300)
        st = S.stats()
        for k, (rid, _) in enumerate(ids):
            out = S.poll(rid)
            assert out is not None
            got[k] = out
        assert st["completed"] == len(reqs) and st["failed"] == 0
        assert st["p50_ms"] > 0 and st["p99_ms"] >= st["p50_ms"] and st["solves_per_s"] > 0
        # arrivals overlapped: some launch held more than one system
        assert st["launches"] < sum(r.outer for r, _ in got.values()) * 1000
    for k, rq in enumerate(reqs):
        r, lat = got[k]
        assert r.done and r.solver_state == lmp.kSolverSuccess, (k, rq, r)
        assert r.res_rel < RTOL and lat > 0
        s = ids[k][1] or P.q1_system(rq["dim"], rq["cells"], rq["seed"], rq["sigma"])
        # host and device assembly agree to a few ulps of the coefficient, so
        # the true residual is checked against the host system with a margin
        assert _true_rel_res(s, r.x) < 1.001 * RTOL, (k, rq)
    # isolation: every fourth request again, alone on a fresh server
    with Server(2, rtol=RTOL, platform=plat) as A:
        for k in range(0, len(reqs), 4):
            rid, _ = _submit(A, reqs[k], k)
            alone, _ = A.wait(rid, 120)
            mixed = got[k][0]
            assert alone.iters == mixed.iters and alone.outer == mixed.outer, k
            np.testing.assert_array_equal(alone.x, mixed.x)


def test_admission_respects_hbm_budget(plat):
    s = P.q1_system(2, 40, 77, 1.0)
    one = slot_bytes(s.n, s.nnz, 9, True)
    budget = int(2.5 * one)
    systems = [P.q1_system(2, 40, 77 + k, 1.0) for k in range(6)]
    with Server(8, rtol=RTOL, hbm_budget=budget, chunk_passes=8, platform=plat) as S:
        ids = [S.submit_system(x) for x in systems]
        S.drain(120)
        st = S.stats()
        assert st["completed"] == 6 and st["hbm_peak"] <= budget and st["hbm_peak"] >= one
        assert st["hbm_in_use"] == 0 and st["running"] == 0
        for rid, x in zip(ids, systems):
            r, _ = S.poll(rid)
            assert r.solver_state == lmp.kSolverSuccess and _true_rel_res(x, r.x) < 1.001 * RTOL
    # a budget two systems fit in: one system larger than it fails at once
    with Server(4, hbm_budget=budget, platform=plat) as S:
        big = P.q1_system(2, 90, 5, 1.0)
        with pytest.raises(lmp.B200LAError) as e:
            S.submit_system(big)
        assert e.value.status == -3


def test_large_request_is_not_starved(plat):
    """The queue head (a large system) waits while small ones run, and is
    admitted after at most max_skips rounds of passing it over."""
    small = [P.q1_system(2, 12, 300 + k, 0.5) for k in range(12)]
    large = P.q1_system(2, 60, 299, 0.5)
    budget = int(1.2 * slot_bytes(large.n, large.nnz, 9, True))
    with Server(16, rtol=RTOL, hbm_budget=budget, chunk_passes=4, max_skips=2, platform=plat) as S:
        first = S.submit_system(small[0])
        lid = S.submit_system(large)
        sids = [S.submit_system(x) for x in small[1:]]
        S.drain(120)
        r, _ = S.poll(lid)
        assert r.solver_state == lmp.kSolverSuccess
        assert all(S.poll(i)[0].solver_state == lmp.kSolverSuccess for i in [first] + sids)


def test_fault_injection_on_the_host(plat):
    with Server(8, rtol=RTOL, platform=plat) as S:
        good = P.q1_system(2, 20, 11, 1.0)
        # malformed CSR: column out of range -> refused at submission
        rp = np.array([0, 2, 3], np.int32)
        with pytest.raises(lmp.B200LAError) as e:
            S.submit(rp, np.array([0, 5, 1], np.int32), np.ones(3), np.ones(2))
        assert e.value.status == -5
        # rowptr not monotone -> refused
        with pytest.raises(lmp.B200LAError) as e:
            S.submit(np.array([0, 3, 2], np.int32), np.array([0, 1, 1], np.int32), np.ones(3), np.ones(2))
        assert e.value.status == -5
        # non-finite right-hand side: runs, ends without success
        bad_b = good.b.copy()
        bad_b[3] = np.nan
        nan_id = S.submit(good.rowptr, good.col, good.val, bad_b)
        # a row without its diagonal: the Jacobi solve ends with an error state
        nodiag = S.submit(np.array([0, 2, 3], np.int32), np.array([0, 1, 0], np.int32),
                          np.array([2.0, 1.0, 1.0]), np.array([1.0, 1.0]))
        ok_id = S.submit_system(good)
        S.drain(120)
        r_nan, _ = S.poll(nan_id)
        assert r_nan.done and r_nan.solver_state != lmp.kSolverSuccess
        r_nd, _ = S.poll(nodiag)
        assert r_nd.done and r_nd.solver_state == lmp.kSolverError
        r_ok, _ = S.poll(ok_id)
        assert r_ok.solver_state == lmp.kSolverSuccess and _true_rel_res(good, r_ok.x) < 1.001 * RTOL
        st = S.stats()
        assert st["completed"] == 3 and st["failed"] == 0
        # release frees the stored solution; the id is then unknown
        S.release(ok_id)
        with pytest.raises(lmp.B200LAError):
            S.poll(ok_id)
