"""Batched / continuously batched PCG on the GPU against the CPU oracle.

* FP64 mode: each system in a mixed batch takes the reference CG's
  iteration count (+-1) and matches the oracle's solution within 1e-10.
* Mixed mode (FP32 inner + FP64 refinement): every system reaches the stated
  FP64 relative residual; its error against the FP64 oracle is bounded.
* Isolation: a system's result is the same alone, in the mix, and when it is
  admitted while other systems are already running (per-system reductions are
  deterministic, so the results agree bit for bit).
"""
import numpy as np
import pytest

import oracle
from ba_b200 import lmp
from ba_b200 import problems as P
from ba_b200.batch import Batch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def plat():
    return lmp.init_platform(0)


def _mix(seed=1, count=12):
    out = []
    for k in range(count):
        dim = 2 if k % 3 else 3
        n = [6, 17, 31, 9, 40, 12][k % 6] if dim == 2 else [4, 7, 10][k % 3]
        sigma = [0.0, 1.0, 2.0][k % 3]
        out.append(P.q1_system(dim, n, seed * 100 + k, sigma, f"mix{k}"))
    return out


def test_fp64_batch_matches_reference_cg(plat):
    systems = _mix()
    B = Batch(len(systems), mixed=False, precond=True, rtol=1e-10, atol=0.0, dtol=1e8, platform=plat)
    slots = [B.add_system(s) for s in systems]
    assert B.run() == 0
    for s, sl in zip(systems, slots):
        r = B.result(sl)
        ref = oracle.cg(s.rowptr, s.col, s.val, s.b, maxits=100000, atol=0.0, rtol=1e-10, dtol=1e8)
        assert r.done and r.solver_state == lmp.kSolverSuccess, (s.name, r)
        assert abs(r.iters - ref.iters) <= 1, (s.name, r.iters, ref.iters)
        assert np.linalg.norm(r.x - ref.x) <= 1e-10 * np.linalg.norm(ref.x), s.name
        np.testing.assert_allclose(r.res_init, ref.res_init, rtol=1e-12)


def test_fp64_batch_plain_cg(plat):
    """Unpreconditioned FP64 CG (the plain comparator).  On sigma <= 1 systems
    the iteration count is the reference's +-1.  On the sigma = 2 systems
    (coefficient contrast ~e^6 without Jacobi scaling) CG's count is
    sensitive to rounding -- the device's FMA rows and tree-ordered dots move
    it by a few iterations, as they do for the single-system device CG -- so
    there the bar is +-5% and the solution within 1e-10 of the oracle's."""
    systems = _mix(seed=2, count=6)
    B = Batch(8, mixed=False, precond=False, rtol=1e-10, atol=0.0, platform=plat)
    slots = [B.add_system(s) for s in systems]
    B.run()
    rows = []
    for s, sl in zip(systems, slots):
        r = B.result(sl)
        ref = oracle.cg(s.rowptr, s.col, s.val, s.b, maxits=100000, atol=0.0, rtol=1e-10, precond=False)
        # single-system device CG on the same matrix, for comparison
        A = lmp.B200_CSR_lMatrix(s.rowptr, s.col, s.val, platform=plat)
        A.set_format(1, 4)
        bv = lmp.B200_lVector.from_numpy(s.b, platform=plat)
        xv = lmp.B200_lVector(s.n, platform=plat)
        cg = lmp.setup_CG_solver(maxits=100000, atol=0.0, rtol=1e-10, dtol=1e8, use_precond=False)
        cg.SetupOperator(A)
        cg.Solve(bv, xv)
        rows.append((s.name, s.n, r.iters, cg.iter(), ref.iters,
                     float(np.linalg.norm(r.x - ref.x) / np.linalg.norm(ref.x))))
    sig = {s.name: s.meta["sigma"] for s in systems}
    bad = [x for x in rows
           if abs(x[2] - x[4]) > (1 if sig[x[0]] <= 1.0 else max(2, 0.05 * x[4])) or x[5] > 1e-10]
    assert not bad, rows


def _true_rel_res(s, x):
    return np.linalg.norm(s.b - oracle.spmv(s.rowptr, s.col, s.val, x)) / np.linalg.norm(s.b)


def test_mixed_batch_reaches_tolerance(plat):
    sizes = P.batch_sizes(24, lo=16, hi=64, seed=5)
    systems = [P.q1_system(2, int(n), 500 + k, 1.0, f"b{k}") for k, n in enumerate(sizes)]
    B = Batch(32, mixed=True, precond=True, rtol=1e-8, platform=plat)
    B.tune()
    slots = [B.add_system(s) for s in systems]
    assert B.run() == 0
    for s, sl in zip(systems, slots):
        r = B.result(sl)
        assert r.done and r.solver_state == lmp.kSolverSuccess, (s.name, r)
        assert r.res_rel < 1e-8
        tr = _true_rel_res(s, r.x)
        assert tr < 1.0001e-8, (s.name, tr)
        ref = oracle.cg(s.rowptr, s.col, s.val, s.b, maxits=100000, atol=0.0, rtol=1e-13)
        err = np.linalg.norm(r.x - ref.x) / np.linalg.norm(ref.x)
        assert err < 1e-5, (s.name, err)
        assert r.outer >= 2 and r.device_us > 0


@pytest.mark.parametrize("restart", [False, True])
def test_mixed_batch_passes_match_oracle(plat, restart):
    """Mixed mode per system against the oracle's restatement of the same
    refinement: with kept directions (default; oracle.mpcg_kept) and
    restarted per pass (oracle.mpir, MPIR's form), both with the batch's
    last-pass floor (an inner pass stops at half the outer target).  Passes within one, inner iterations within 10% (the device's
    FP32 dots are compensated and tree-ordered, the oracle's are the
    reference's grouped sums), FP64 true residual at the tolerance."""
    systems = _mix(seed=7, count=9)
    irt = 1e-4 if restart else 0.1
    B = Batch(16, mixed=True, precond=True, rtol=1e-9, inner_rtol=irt, restart_inner=restart, max_outer=40,
              platform=plat)
    slots = B.add_many([(s.rowptr, s.col, s.val, s.b) for s in systems])
    B.solve()
    rows = []
    for s, r in zip(systems, B.results(slots)):
        if restart:
            ref, passes = oracle.mpir(s.rowptr, s.col, s.val, s.b, rtol=1e-9, inner_rtol=irt, max_outer=40,
                                      floor=0.5)
        else:
            ref, passes = oracle.mpcg_kept(s.rowptr, s.col, s.val, s.b, rtol=1e-9, inner_rtol=irt, max_outer=40,
                                           floor=0.5)
        assert r.solver_state == lmp.kSolverSuccess and ref.state == 0, (s.name, r)
        assert _true_rel_res(s, r.x) < 1.0001e-9, s.name
        rows.append((s.name, r.outer, passes, r.iters, ref.iters))
    bad = [x for x in rows if abs(x[1] - x[2]) > 1 or abs(x[3] - x[4]) > max(3, 0.1 * x[4])]
    assert not bad, rows


def test_isolation_alone_vs_mix_vs_late_admission(plat):
    systems = _mix(seed=3, count=9)
    probe = systems[4]
    kw = dict(mixed=True, precond=True, rtol=1e-9, platform=plat)
    # alone
    A = Batch(1, **kw)
    a = A.add_system(probe)
    A.run()
    alone = A.result(a)
    # in the mix
    M = Batch(16, **kw)
    slots = [M.add_system(s) for s in systems]
    M.run()
    mixed = M.result(slots[4])
    # admitted while the others are running (continuous batching)
    L = Batch(16, **kw)
    others = [L.add_system(s) for k, s in enumerate(systems) if k != 4]
    assert L.run(max_passes=7) > 0
    late = L.add_system(probe)
    while L.run(max_passes=5) > 0:
        pass
    late_r = L.result(late)
    for r in (mixed, late_r):
        assert r.iters == alone.iters and r.outer == alone.outer
        np.testing.assert_array_equal(r.x, alone.x)
    for k, sl in zip([k for k in range(9) if k != 4], others):
        r = L.result(sl)
        np.testing.assert_array_equal(r.x, M.result(slots[k]).x)


def test_slots_capacity_remove_and_bad_diagonal(plat):
    B = Batch(2, mixed=False, rtol=1e-10, atol=0.0, platform=plat)
    s = P.poisson_2d(8)
    a = B.add_system(s)
    b = B.add_system(s)
    with pytest.raises(lmp.B200LAError):
        B.add_system(s)
    B.run()
    B.remove(a)
    used, nbytes = B.info()
    assert used == 1 and nbytes > 0
    # a row without a diagonal: the Jacobi solve ends with an error state
    rowptr = np.array([0, 2, 3], np.int32)
    col = np.array([0, 1, 0], np.int32)
    c = B.add(rowptr, col, np.array([2.0, 1.0, 1.0]), np.array([1.0, 1.0]))
    B.run()
    r = B.result(c)
    assert r.done and r.solver_state == lmp.kSolverError
    assert B.result(b).solver_state == lmp.kSolverSuccess


@pytest.mark.parametrize("dim,cells,sigma", [(2, 9, 0.0), (2, 33, 1.0), (3, 6, 0.0), (3, 11, 2.0)])
def test_device_assembly_matches_host_generator(plat, dim, cells, sigma):
    """The device-built Q1 system equals ba_b200.problems' host system:
    structure and RHS bit for bit, values bit for bit for sigma = 0 and within
    a few ulps of the coefficient for sigma > 0 (device exp/log/cos)."""
    B = Batch(2, mixed=True, platform=plat)
    slot = B.add_q1(dim, cells, 4321, sigma)
    rp, cl, vv, bb = B.get_system(slot)
    s = P.q1_system(dim, cells, 4321, sigma)
    np.testing.assert_array_equal(rp, s.rowptr)
    np.testing.assert_array_equal(cl, s.col)
    np.testing.assert_array_equal(bb, s.b)
    if sigma == 0.0:
        np.testing.assert_array_equal(vv, s.val)
    else:
        np.testing.assert_allclose(vv, s.val, rtol=1e-13, atol=1e-300)
    B.run()
    r = B.result(slot)
    assert r.done and r.solver_state == lmp.kSolverSuccess
    assert _true_rel_res(s, r.x) < 1.001e-8


def test_malformed_csr_is_refused_on_the_device_check(plat):
    """batch_add checks the uploaded structure on the device (the checks of
    csr_upload): a bad system returns B200LA_ERR_MATRIX and leaves no slot
    behind; the batch keeps working."""
    B = Batch(4, mixed=True, rtol=1e-8, platform=plat)
    good = P.q1_system(2, 12, 9, 1.0)
    bad_cases = [
        (np.array([0, 2, 3], np.int32), np.array([0, 5, 1], np.int32)),   # column out of range
        (np.array([0, 3, 2], np.int32), np.array([0, 1, 1], np.int32)),   # rowptr decreases
        (np.array([1, 2, 3], np.int32), np.array([0, 1, 1], np.int32)),   # rowptr[0] != 0
        (np.array([0, 1, 7], np.int32), np.array([0, 1, 1], np.int32)),   # rowptr[n] != nnz
    ]
    for rp, cl in bad_cases:
        with pytest.raises(lmp.B200LAError) as e:
            B.add(rp, cl, np.ones(cl.shape[0]), np.ones(2))
        assert e.value.status == -5, e.value
        assert B.info()[0] == 0
    s = B.add_system(good)
    assert B.info()[0] == 1
    B.solve()
    r = B.results([s])[0]
    assert r.solver_state == lmp.kSolverSuccess and _true_rel_res(good, r.x) < 1.001e-8


def test_add_many_matches_single_adds_and_reports_per_system_status(plat):
    """The bulk add gives each system the result it gets from a single add
    (bit for bit) and reports a malformed one on its own."""
    systems = _mix(seed=4, count=5)
    A = Batch(8, mixed=True, rtol=1e-8, platform=plat)
    one = [A.add_system(s) for s in systems]
    A.solve()
    M = Batch(8, mixed=True, rtol=1e-8, platform=plat)
    bad = (np.array([0, 2, 3], np.int32), np.array([0, 9, 1], np.int32), np.ones(3), np.ones(2))
    items = [(s.rowptr, s.col, s.val, s.b) for s in systems]
    items.insert(2, bad)
    with pytest.raises(lmp.B200LAError) as e:
        M.add_many(items)
    assert e.value.status == -5
    assert M.last_status == [0, 0, -5, 0, 0, 0]
    assert M.last_slots[2] == -1 and M.info()[0] == 5
    M.solve()
    good = [sl for sl in M.last_slots if sl >= 0]
    for a_slot, rm in zip(one, M.results(good)):
        ra = A.results([a_slot])[0]
        assert rm.solver_state == lmp.kSolverSuccess
        np.testing.assert_array_equal(ra.x, rm.x)


def test_large_system_ticket_path_isolated_and_converged(plat):
    # 128-row items: the 3D system has 2,350 items in K1 and K2 (more than
    # kDirectItems = 1,024), so its p.Ap and r.r/r.z totals go through the
    # two-level last-arriver tickets (36 full groups of 64 items and one of
    # 46, then the system's 37 group sums), while the small systems re-add
    # their partials.
    big = P.q1_system(3, 66, 77, 1.0, "big3d_66")
    small = [P.q1_system(2, c, 500 + c, 1.0, f"s{c}") for c in (9, 30, 64)]
    kw = dict(mixed=True, precond=True, rtol=1e-8, platform=plat)
    A = Batch(1, **kw)
    A.set_items(128, 128, 256, adaptive=False)
    a = A.add_system(big)
    A.run()
    alone = A.result(a)
    M = Batch(8, **kw)
    M.set_items(128, 128, 256, adaptive=False)
    slots = [M.add_system(s) for s in small[:2]] + [M.add_system(big)] + [M.add_system(small[2])]
    M.run()
    mixed = M.result(slots[2])
    assert alone.solver_state == lmp.kSolverSuccess
    assert mixed.iters == alone.iters and mixed.outer == alone.outer
    np.testing.assert_array_equal(mixed.x, alone.x)
    res = np.linalg.norm(big.b - oracle.spmv(big.rowptr, big.col, big.val, alone.x))
    assert res <= 1.001e-8 * np.linalg.norm(big.b)
    for s, sl in zip(small[:2] + small[2:], slots[:2] + slots[3:]):
        r = M.result(sl)
        assert r.solver_state == lmp.kSolverSuccess
        assert np.linalg.norm(s.b - oracle.spmv(s.rowptr, s.col, s.val, r.x)) <= 1.001e-8 * np.linalg.norm(s.b)


def test_adds_overlapping_launches_match_the_plain_solve(plat):
    # systems added in chunks while earlier chunks already iterate (adds on the
    # batch's transfer stream, launches asynchronous) end bit for bit as when
    # all are added first: a system's arithmetic does not depend on when it
    # joined or on what else runs
    systems = _mix(seed=5, count=12)
    kw = dict(mixed=True, precond=True, rtol=1e-9, platform=plat)
    A = Batch(16, **kw)
    A.set_items(128, 512, 512, adaptive=False)
    slots_a = A.add_many([(s.rowptr, s.col, s.val, s.b) for s in systems])
    A.solve(16)
    ref = A.results(slots_a)
    B = Batch(16, **kw)
    B.set_items(128, 512, 512, adaptive=False)
    order = sorted(range(len(systems)), key=lambda k: -systems[k].n)
    slot_of = {}
    for c in range(0, len(order), 4):
        chunk = order[c:c + 4]
        for k, sl in zip(chunk, B.add_many([(systems[k].rowptr, systems[k].col, systems[k].val, systems[k].b)
                                            for k in chunk])):
            slot_of[k] = sl
        B.launch(8)
    B.solve(16)
    got = B.results([slot_of[k] for k in range(len(systems))])
    for k, (r, g) in enumerate(zip(ref, got)):
        assert g.solver_state == lmp.kSolverSuccess, (k, g)
        assert (g.iters, g.outer) == (r.iters, r.outer)
        np.testing.assert_array_equal(g.x, r.x)


def test_initial_guesses_in_one_add_many(plat):
    # one add_many call mixing systems with an initial guess (copied to x) and
    # without (x zeroed by the setup kernel): the latter repeat a plain run bit
    # for bit, the former start from their guess (res_init is its residual)
    # and reach the tolerance relative to it
    sizes = P.batch_sizes(8, lo=16, hi=48, seed=9)
    systems = [P.q1_system(2, int(n), 900 + k, 1.0, f"g{k}") for k, n in enumerate(sizes)]
    kw = dict(mixed=True, precond=True, rtol=1e-8, platform=plat)
    A = Batch(8, **kw)
    sa = A.add_many([(s.rowptr, s.col, s.val, s.b) for s in systems])
    A.solve(16)
    ra = A.results(sa)
    guesses = [r.x * (1.0 + 1e-3) if k % 2 == 0 else None for k, r in enumerate(ra)]
    B = Batch(8, **kw)
    sb = B.add_many([(s.rowptr, s.col, s.val, s.b, g) for s, g in zip(systems, guesses)])
    B.solve(16)
    rb = B.results(sb)
    for k, (s, a, b, g) in enumerate(zip(systems, ra, rb, guesses)):
        assert b.done and b.solver_state == lmp.kSolverSuccess, (s.name, b)
        if g is None:
            assert b.iters == a.iters and np.array_equal(b.x, a.x), s.name
            continue
        r0 = np.linalg.norm(s.b - oracle.spmv(s.rowptr, s.col, s.val, g))
        assert abs(b.res_init - r0) <= 1e-9 * r0, (s.name, b.res_init, r0)
        assert b.res_init < 1e-2 * a.res_init
        assert np.linalg.norm(s.b - oracle.spmv(s.rowptr, s.col, s.val, b.x)) <= 1.0001e-8 * r0, s.name
    A.close()
    B.close()


def test_registered_outputs_are_copied_as_systems_finish(plat):
    # solutions registered with set_outputs are copied out on the transfer
    # stream when a run sees their system finished; results(out=...) then
    # only waits.  They equal the plain read bit for bit; status-only reads
    # keep a registration, a restart ends them all.
    import torch
    sizes = P.batch_sizes(12, lo=16, hi=96, seed=21)
    systems = [P.q1_system(2, int(n), 40 + k, 1.0, f"o{k}") for k, n in enumerate(sizes)]
    kw = dict(mixed=True, precond=True, rtol=1e-8, platform=plat)
    A = Batch(12, **kw)
    sa = A.add_many([(s.rowptr, s.col, s.val, s.b) for s in systems])
    A.solve(8)
    ra = A.results(sa)
    B = Batch(12, **kw)
    sb = B.add_many([(s.rowptr, s.col, s.val, s.b) for s in systems])
    outs = [torch.empty(s.n, dtype=torch.float64).pin_memory().numpy() for s in systems]
    B.set_outputs(sb, outs)
    B.run(20)
    for sl in sb:
        B.result(sl, with_x=False)  # status-only reads keep the registrations
    B.solve(8)  # small launches: most systems finish, and are copied, before the last one
    rb = B.results(sb, out=outs)
    for a, b, o in zip(ra, rb, outs):
        assert b.x is o and np.array_equal(b.x, a.x) and b.iters == a.iters
    B.restart()
    B.solve(8)
    rc = B.results(sb)
    for a, c in zip(ra, rc):
        assert np.array_equal(c.x, a.x)
    with pytest.raises(lmp.B200LAError):
        B.set_outputs([sb[0]], [np.empty(3)])
    A.close()
    B.close()


def test_remove_many(plat):
    sizes = P.batch_sizes(6, lo=16, hi=32, seed=3)
    systems = [P.q1_system(2, int(n), 70 + k, 1.0, f"r{k}") for k, n in enumerate(sizes)]
    B = Batch(6, mixed=True, precond=True, rtol=1e-8, platform=plat)
    sl = B.add_many([(s.rowptr, s.col, s.val, s.b) for s in systems])
    used0, bytes0 = B.info()
    # a bad list frees nothing: a repeated slot, a free slot
    for bad in ([sl[0], sl[0]], [sl[1], 99]):
        with pytest.raises(lmp.B200LAError):
            B.remove_many(bad)
    assert B.info() == (used0, bytes0)
    B.remove_many([sl[1], sl[2], sl[4]])
    used1, bytes1 = B.info()
    assert used1 == used0 - 3 and bytes1 < bytes0
    # the freed slots take new systems, and every system still solves alone
    again = B.add_many([(systems[k].rowptr, systems[k].col, systems[k].val, systems[k].b) for k in (1, 2, 4)])
    B.solve(16)
    ref = Batch(1, mixed=True, precond=True, rtol=1e-8, platform=plat)
    one = ref.add_system(systems[2])
    ref.solve(16)
    r = B.results([again[1]])[0]
    assert np.array_equal(r.x, ref.result(one).x)
    B.close()
    ref.close()


def test_remove_and_reuse_slots_while_a_launch_is_in_flight(plat):
    # running systems are removed while an asynchronous launch is in flight and
    # new systems are added into the freed slots at once.  The removal clears
    # the slots' states on the solve stream after the launch; the adds run on
    # the transfer stream and must be ordered after that, or a new system's
    # fresh state would be cleared (it would never solve) and the running
    # kernels would read its descriptor.  Each new system, and the survivor,
    # must end with the bits it gets when solved alone.
    first = [P.q1_system(2, c, 300 + k, 1.0, f"f{k}") for k, c in enumerate((160, 200, 180, 220))]
    second = [P.q1_system(2, c, 400 + k, 1.0, f"s{k}") for k, c in enumerate((40, 64, 90))]
    kw = dict(mixed=True, precond=True, rtol=1e-8, platform=plat)

    def alone(s):
        A = Batch(1, **kw)
        A.set_items(128, 512, 512, adaptive=False)
        a = A.add_system(s)
        A.solve(16)
        r = A.result(a)
        A.close()
        return r

    B = Batch(4, **kw)
    B.set_items(128, 512, 512, adaptive=False)
    sl = B.add_many([(s.rowptr, s.col, s.val, s.b) for s in first])
    B.launch(200)  # returns at once: the launch is still running below
    gone = [sl[0], sl[1], sl[3]]
    B.remove_many(gone)
    new = B.add_many([(s.rowptr, s.col, s.val, s.b) for s in second])
    assert sorted(new) == sorted(gone)
    B.solve(16)
    got = B.results(new + [sl[2]])
    for s, g in zip(second + [first[2]], got):
        ref = alone(s)
        assert g.done and g.solver_state == lmp.kSolverSuccess, (s.name, g)
        assert (g.iters, g.outer) == (ref.iters, ref.outer), s.name
        np.testing.assert_array_equal(g.x, ref.x)
    assert B.info()[0] == 4
    B.close()


@pytest.mark.parametrize("mixed", [True, False])
def test_column_storages_give_the_same_bits(plat, mixed):
    # the sliced copy stores no columns (values-only stencil layout, Q1
    # systems), int16 offsets or int32 columns: each row adds the same
    # products in the same order whatever the storage, so every system --
    # uploaded CSR (stencil found by the device check), device-assembled Q1
    # (stencil known), and a random matrix (no stencil) -- ends bit for bit
    # the same in all three
    systems = _mix(seed=9, count=9) + [P.random_spd(300, 4, density=0.02)]
    q1 = [(2, 37, 5, 1.0), (3, 9, 6, 2.0), (2, 3, 7, 0.5)]
    out = {}
    for bits in (0, 16, 32):
        B = Batch(16, mixed=mixed, precond=True, rtol=1e-9, index_bits=bits, platform=plat)
        B.set_items(128, 512, 512, adaptive=False)
        slots = B.add_many([(s.rowptr, s.col, s.val, s.b) for s in systems])
        slots += [B.add_q1(*a) for a in q1]
        B.solve(16)
        out[bits] = B.results(slots)
        B.close()
    for k in range(len(out[0])):
        for bits in (16, 32):
            a, b = out[0][k], out[bits][k]
            assert a.solver_state == lmp.kSolverSuccess and (a.iters, a.outer) == (b.iters, b.outer), (k, bits)
            np.testing.assert_array_equal(a.x, b.x)
