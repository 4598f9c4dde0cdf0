"""Multi-rank CoupledVector / CoupledMatrix / CG host logic (ba_b200.coupled)
on CPU: thread ranks and world_size-2 gloo process groups, with host vectors
over the CPU oracle (tests/numpy_lmp.py).  The row-partitioned CG must take
the single-rank reference CG's iteration count (+-1) and match its solution
within 1e-10; the coupled SpMV must equal the global one up to the summation
order of the split rows."""
import os
import threading

import numpy as np
import pytest

import oracle
from ba_b200 import coupled as CP
from ba_b200 import problems as P
from tests.numpy_lmp import numpy_backend


def _system():
    return P.q1_system(2, 30, 17, 1.0, "coupled_q1")


def test_split_rows_rebuilds_the_rows():
    s = _system()
    cp = CP.LaCouplings.balanced(s.n, 3)
    for r in range(3):
        b, e = int(cp.offsets[r]), int(cp.offsets[r + 1])
        (drp, dc, dv), (orp, oc, ov), ghosts = CP.split_rows(s.rowptr, s.col, s.val, b, e)
        assert np.all((ghosts < b) | (ghosts >= e)) and np.all(np.diff(ghosts) > 0)
        for i in range(e - b):
            row = s.rowptr[b + i], s.rowptr[b + i + 1]
            want = dict(zip(s.col[row[0]:row[1]], s.val[row[0]:row[1]]))
            got = dict(zip(dc[drp[i]:drp[i + 1]] + b, dv[drp[i]:drp[i + 1]]))
            got.update(zip(ghosts[oc[orp[i]:orp[i + 1]]], ov[orp[i]:orp[i + 1]]))
            assert got == want


def _rank_work(comm, s, results, precond=True):
    make_matrix, make_vector = numpy_backend()
    cp = CP.LaCouplings.balanced(s.n, comm.size)
    A = CP.CoupledMatrix(comm, cp, s.rowptr, s.col, s.val, make_matrix, make_vector)
    b0, e0 = int(cp.offsets[comm.rank]), int(cp.offsets[comm.rank + 1])
    # coupled SpMV of a seeded vector
    xg = P.uniform01(5, s.n, stream=3)
    x, y = A.vector(), A.vector()
    x.interior.a[:] = xg[b0:e0]
    A.VectorMult(x, y)
    b, sol = A.vector(), A.vector()
    b.interior.a[:] = s.b[b0:e0]
    r = CP.coupled_cg(A, b, sol, maxits=5000, atol=0.0, rtol=1e-10, dtol=1e8, precond=precond)
    results[comm.rank] = (y.interior.a.copy(), sol.interior.a.copy(), r)


@pytest.mark.parametrize("size", [1, 2, 3, 4])
@pytest.mark.parametrize("precond", [True, False])
def test_thread_ranks_match_single_rank_cg(size, precond):
    s = _system()
    world = CP.ThreadComm.World(size)
    results = {}
    threads = [threading.Thread(target=_rank_work, args=(world.comm(r), s, results, precond)) for r in range(size)]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=120)
    assert len(results) == size
    y = np.concatenate([results[r][0] for r in range(size)])
    x = np.concatenate([results[r][1] for r in range(size)])
    yg = oracle.spmv(s.rowptr, s.col, s.val, P.uniform01(5, s.n, stream=3))
    np.testing.assert_allclose(y, yg, rtol=1e-13, atol=1e-15)
    ref = oracle.cg(s.rowptr, s.col, s.val, s.b, maxits=5000, atol=0.0, rtol=1e-10, precond=precond)
    its = {results[r][2].iters for r in range(size)}
    assert len(its) == 1 and abs(its.pop() - ref.iters) <= 1
    assert np.linalg.norm(x - ref.x) <= 1e-10 * np.linalg.norm(ref.x)


def _gloo_rank(rank, size, port, out_dir):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=size)
    try:
        comm = CP.TorchComm()
        results = {}
        _rank_work(comm, _system(), results)
        y, x, r = results[rank]
        np.savez(os.path.join(out_dir, f"r{rank}.npz"), y=y, x=x, iters=r.iters, state=r.state)
    finally:
        dist.destroy_process_group()


def test_gloo_two_ranks_match_single_rank_cg(tmp_path):
    import torch.multiprocessing as mp
    import socket
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    mp.start_processes(_gloo_rank, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    parts = [np.load(tmp_path / f"r{r}.npz") for r in range(2)]
    s = _system()
    x = np.concatenate([p["x"] for p in parts])
    ref = oracle.cg(s.rowptr, s.col, s.val, s.b, maxits=5000, atol=0.0, rtol=1e-10)
    assert int(parts[0]["iters"]) == int(parts[1]["iters"])
    assert abs(int(parts[0]["iters"]) - ref.iters) <= 1
    assert np.linalg.norm(x - ref.x) <= 1e-10 * np.linalg.norm(ref.x)
