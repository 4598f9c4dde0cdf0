"""Multi-rank CoupledMatrix / CoupledVector / CG (ba_b200.coupled) with the
B200 backend on one GPU: the ranks run as threads of this process, each with
its own device context and stream (ThreadComm), so no kernel waits on another
rank's kernel.  The diagonal and off-diagonal blocks are B200 CSR matrices.
The halo runs host-staged (the device vectors' GetValues/SetValues around a
host exchange) or device-resident (gather kernel into a device send buffer,
device-to-device copies between the ranks' buffers, scatter kernel into the
ghost vector).  Bar: the single-rank reference CG's iteration count (+-1) and
solution within 1e-10; the coupled SpMV equal to the global product up to
summation order; both halo forms give the same bits."""
import threading

import numpy as np
import pytest

import oracle
from ba_b200 import coupled as CP
from ba_b200 import lmp
from ba_b200 import problems as P

pytestmark = pytest.mark.gpu


def _rank(comm, s, out, precond):
    plat = lmp.Platform(0)
    make_matrix, make_vector = CP.device_backend(plat)
    cp = CP.LaCouplings.balanced(s.n, comm.size)
    A = CP.CoupledMatrix(comm, cp, s.rowptr, s.col, s.val, make_matrix, make_vector)
    b0, e0 = int(cp.offsets[comm.rank]), int(cp.offsets[comm.rank + 1])
    x, y = A.vector(), A.vector()
    x.interior.SetBlockValues(0, e0 - b0, P.uniform01(5, s.n, stream=3)[b0:e0])
    A.VectorMult(x, y)
    b, sol = A.vector(), A.vector()
    b.interior.SetBlockValues(0, e0 - b0, s.b[b0:e0])
    r = CP.coupled_cg(A, b, sol, maxits=5000, atol=0.0, rtol=1e-10, dtol=1e8, precond=precond)
    out[comm.rank] = (y.interior.numpy(), sol.interior.numpy(), r)


def _run(size, s, precond, device_halo):
    world = CP.ThreadComm.World(size)
    out, errors = {}, []

    def run(r):
        try:
            _rank(world.comm(r, device_halo=device_halo), s, out, precond)
        except BaseException as e:  # surface the rank's error in the test
            errors.append(e)
            world.barrier.abort()

    threads = [threading.Thread(target=run, args=(r,)) for r in range(size)]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=300)
    assert not errors, errors
    return out


@pytest.mark.parametrize("size", [2, 3])
@pytest.mark.parametrize("precond", [True, False])
@pytest.mark.parametrize("device_halo", [False, True])
def test_device_ranks_match_single_rank_cg(size, precond, device_halo):
    s = P.q1_system(3, 12, 31, 1.0, "coupled3d")
    out = _run(size, s, precond, device_halo)
    y = np.concatenate([out[r][0] for r in range(size)])
    x = np.concatenate([out[r][1] for r in range(size)])
    yg = oracle.spmv(s.rowptr, s.col, s.val, P.uniform01(5, s.n, stream=3))
    np.testing.assert_allclose(y, yg, rtol=1e-13, atol=1e-15)
    ref = oracle.cg(s.rowptr, s.col, s.val, s.b, maxits=5000, atol=0.0, rtol=1e-10, precond=precond)
    its = {out[r][2].iters for r in range(size)}
    assert len(its) == 1 and abs(its.pop() - ref.iters) <= 1
    assert np.linalg.norm(x - ref.x) <= 1e-10 * np.linalg.norm(ref.x)


def test_device_halo_gives_the_host_halos_bits():
    s = P.q1_system(2, 30, 17, 1.0, "coupled2d")
    a = _run(3, s, True, False)
    b = _run(3, s, True, True)
    for r in range(3):
        np.testing.assert_array_equal(a[r][0], b[r][0])
        np.testing.assert_array_equal(a[r][1], b[r][1])
        assert a[r][2].iters == b[r][2].iters
