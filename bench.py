#!/usr/bin/env python
"""Benchmark of the PCG hot path on B200: one JSON line on rank 0.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload batch|poisson3d|varcoef3d|serve|bicgstab|jacobi|gmres|coo]

Workload "batch" (default): 1,024 independent 2D Q1 diffusion systems, n x n
cells with n log-uniform in [16, 256] from the seed, lognormal per-cell
coefficient (sigma = 1), seeded U[0,1) RHS, solved to 1e-8 relative FP64
residual by FP32 Jacobi-PCG inside FP64 refinement, all systems in one
CUDA-graph launch with the tuned SpMV schedule.  A step solves the whole
batch; the metric is solves/s, with p50/p99 of the per-system device latency
inside the step.  The plain FP64 GPU CG comparator solves the same batch with
the unpreconditioned FP64 CG recurrence.  The batch's matrices (about 1.3 GB
of FP64 CSR) are larger than L2.

Workload "poisson3d": FP64 Jacobi-PCG on 3D Q1 Poisson, 128^3 cells
(2,146,689 DOFs, 57,066,625 nnz), rel. 1e-10; a step is one solve.
Workload "varcoef3d": the same shape with a lognormal coefficient (sigma 2),
FP32 PCG inside FP64 refinement to 1e-10.  Workload "serve": a seeded
Poisson-arrival request stream through the request loop (p50/p99).
Workloads "bicgstab", "gmres" and "jacobi": the poisson3d matrix solved by
FP64 BiCGSTAB and by GMRES(100), both with right Jacobi preconditioning, to
1e-10 (solves/s), and swept by the Jacobi smoother (100 sweeps per step,
sweeps/s).  Workload "coo": TransformFromCOO of the same matrix from 57M
shuffled triplets (conversions/s).

Multi-GPU: every rank solves its own batch (seeded per rank): independent
systems need no exchange, value = all ranks' solves / the slowest rank's time.

--impl reference times the reference's own CPU implementation (HiFlow3 lmp
sources compiled into oracle/_ref: OPENMP CSR SpMV on all host cores, lmp
BLAS-1, lPreconditioner_Jacobi, the CG<LAD> call sequence; the reference has
no mixed-precision GPU path) on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from ba_b200 import dist as D  # noqa: E402  (host-side helpers only; no CUDA at import)

METRIC = "PCG solves/s & p50/p99 latency at 1e-8 rel. residual vs plain FP64 GPU CG"
COUNTS = os.path.join(ROOT, "tests", "golden", "workload_counts.json")
BATCH_COUNT = 1024
BATCH_RTOL = 1e-8
CHUNK = 64  # device-loop passes per graph launch (item lists compacted in between)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="batch",
                    choices=["batch", "poisson3d", "varcoef3d", "serve", "bicgstab", "jacobi", "gmres", "coo"])
    ap.add_argument("--cells", type=int, default=128, help="poisson3d cells per axis")
    ap.add_argument("--count", type=int, default=BATCH_COUNT, help="batch: systems per step")
    ap.add_argument("--requests", type=int, default=64, help="serve: requests per timed step")
    ap.add_argument("--latency-requests", type=int, default=256, help="serve: requests of the latency stream")
    ap.add_argument("--load", type=float, default=0.7,
                    help="serve: Poisson arrival rate of the latency stream, as a fraction of measured throughput")
    ap.add_argument("--hi-dofs", type=float, default=2e6, help="serve: largest request (DOFs)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--inner-rtol", type=float, default=None,
                    help="mixed precision: reduction of an inner pass before the FP64 residual replaces it "
                         "(default: 0.1)")
    ap.add_argument("--split", action="store_true",
                    help="batch: partition ONE 1,024-system batch over the ranks by nnz (greedy, largest first; "
                         "strong scaling) instead of one seeded batch per rank (weak scaling); serve: route ONE "
                         "request stream (N times the requests) over the ranks, join-shortest-queue by "
                         "outstanding nonzeros")
    ap.add_argument("--full-stream", action="store_true",
                    help="serve: also serve the whole seeded request stream at the latency stream's arrival rate")
    ap.add_argument("--stream-count", type=int, default=20000, help="serve --full-stream: requests of the stream")
    return ap.parse_args()


def work_stream(torch):
    """A non-default CUDA stream made torch's current one: the library's
    context runs its work on it (b200la_ctx_set_stream), so the CUDA events
    recorded on it time the device work itself.  (Handing the library the
    legacy default stream, handle 0, would select the context's own stream,
    which the events on stream 0 do not wait for.)"""
    st = torch.cuda.Stream()
    torch.cuda.set_stream(st)
    return st


def dist_env():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0")),
            int(os.environ.get("WORLD_SIZE", "1")))


def measured_peak_gbs():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        return float(json.load(open(p))["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def dram_rate(traffic, kernel_ms, peak):
    """The dominant kernel's physical DRAM rate: the ncu-measured traffic per
    launch over the CUDA-event duration (null without a capture).  Compressed
    storage (int16 column offsets, no row pointer) moves fewer bytes than the
    algorithmic count, so this can sit below `frac`."""
    if not traffic or not kernel_ms:
        return {"traffic_gbs": None, "traffic_frac": None}
    gbs = traffic / (kernel_ms * 1e-3) / 1e9
    return {"traffic_gbs": gbs, "traffic_frac": gbs / peak}


def profile_traffic(key):
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(p):
        return json.load(open(p)).get(key)
    return None


class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, local_rank: int):
        vis = os.environ.get("CUDA_VISIBLE_DEVICES")
        self.index = vis.split(",")[local_rank] if vis else str(local_rank)
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", self.index], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (FileNotFoundError, OSError):
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        self.proc.wait()
        sm, smax, reasons, n = [], [], set(), 0
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            n += 1
            for k, nm in enumerate(names):
                if f[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": n}


def spmv_bytes(n: int, nnz: int, sv: int) -> int:
    """Algorithmic bytes of one SpMV: values+indices, row pointer, x read once, y written."""
    return nnz * (sv + 4) + (n + 1) * 4 + n * sv + n * sv


# ----------------------------------------------------------------- batch workload
def batch_seed(rank: int) -> int:
    from ba_b200 import problems as P
    return D.rank_seed(P.SEED_BATCH, rank)


def make_batch_systems(count: int, rank: int):
    from ba_b200 import problems as P
    return P.batch_systems(count, sigma=1.0, seed=batch_seed(rank))


# The CPU legs (the reference arm and the GPU line's cpu_baseline) time the
# same fixed sample of the batch: BATCH_CPU_SAMPLE systems stratified by size
# (problems.stratified_sample over nnz), so its mean cost per system tracks
# the whole batch's.  The same 32 systems are the ones whose solutions the
# reference recorded for the error statement (reference_fullsize_solutions.json).
BATCH_CPU_SAMPLE = 32


def batch_cpu_sample(systems):
    from ba_b200 import problems as P
    return P.stratified_sample([s.nnz for s in systems], BATCH_CPU_SAMPLE)


def ref_batch_sample(systems, pick, nthreads: int):
    """The reference's CPU CG (FP64 Jacobi-PCG, OPENMP SpMV) to 1e-8 on the
    given systems of the batch; returns (solves, seconds)."""
    import oracle
    total = 0.0
    for i in pick:
        s = systems[int(i)]
        ref = oracle.RefSystem(s.rowptr, s.col, s.val, impl=oracle.IMPL_OPENMP, nthreads=nthreads)
        _, sec = ref.cg(s.b, maxits=100000, atol=0.0, rtol=BATCH_RTOL, dtol=1e8, precond=True)
        ref.close()
        total += sec
    return len(pick), total


def batch_solver_bytes(systems, results) -> int:
    """Algorithmic HBM bytes of the whole mixed-precision batch solve: per
    FP32 inner iteration 8*nnz + 4(n+1) (SpMV: values, indices, row pointer)
    + 8n (p gathered once, Ap written) + 16n (update: read r,Ap,invD, write r)
    + 24n (correction and direction: read p,c,r,invD, write c,p); per
    refinement pass 12*nnz + 4(n+1) + 16n (FP64 residual SpMV: x once, b)
    + 8n (write r, c) + 16n (new direction: read r,invD,p, write p) + 24n
    (x += c + alpha p at the pass's end)."""
    total = 0
    for s, r in zip(systems, results):
        n, nnz = s.n, s.nnz
        total += r.iters * (8 * nnz + 4 * (n + 1) + 48 * n)
        total += (r.outer + 1) * (12 * nnz + 4 * (n + 1) + 64 * n)
    return int(total)


def batch_config(args, systems):
    """The workload, identical in both arms; how each arm computes it goes
    under the line's "details"."""
    n_tot = int(sum(s.n for s in systems))
    nnz_tot = int(sum(s.nnz for s in systems))
    return {"workload": f"batched: {len(systems)} independent 2D Q1 systems, n~logU[16,256] cells, "
                        f"lognormal kappa sigma=1, rel. residual 1e-8",
            "systems": len(systems), "dofs_total": n_tot, "nnz_total": nnz_tot,
            "l2": "inputs larger than L2 (per batch: 1.4 GB FP64 CSR as uploaded, 0.47 GB FP32 and 0.93 GB "
                  "FP64 sliced values)"}


def batch_cpu_sample_text(args, pick, nthreads):
    return (f"the same {len(pick)} systems of the {args.count}-system batch every step (stratified by nnz: "
            f"the middle system of each of {len(pick)} equal-count size strata), each solved to 1e-8 by "
            f"HiFlow3 lmp CG (FP64 Jacobi-PCG, OPENMP SpMV, {nthreads} threads)")


def run_reference_batch(args, rank):
    import oracle
    if not oracle.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built (reference sources absent)"}))
        return
    systems = make_batch_systems(args.count, 0)
    pick = batch_cpu_sample(systems)
    nthreads = os.cpu_count() or 1
    rates, secs = [], []
    for step in range(args.warmup + args.steps):
        cnt, sec = ref_batch_sample(systems, pick, nthreads)
        if step >= args.warmup:
            rates.append(cnt / sec)
            secs.append(sec)
    value = statistics.median(rates)
    sample = batch_cpu_sample_text(args, pick, nthreads)
    out = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup,
        # the wall time each timed step actually took (the sample's solves)
        "ms_per_step": 1e3 * statistics.median(secs),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": batch_config(args, systems),
        "details": {"parallelism": f"cpu openmp x{nthreads}",
                    "precision": "FP64 Jacobi-PCG (the reference's CPU path)",
                    "step": sample,
                    "full_batch_ms_extrapolated": 1e3 * args.count / value},
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": nthreads, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out))


FULLSIZE = os.path.join(ROOT, "tests", "golden", "reference_fullsize_solutions.json")


def fullsize_fixture():
    """The reference's recorded solutions (fingerprints) of the full-size
    workloads, or {} if absent."""
    return json.load(open(FULLSIZE)) if os.path.exists(FULLSIZE) else {}


def batch_error_vs_cpu_oracle(systems, results):
    """Error of the batch's solutions of the stratified sample against the
    reference's FP64 CPU CG to 1e-12 (recorded fingerprints); None when the
    batch is not the recorded one."""
    from ba_b200 import problems as P
    rec = fullsize_fixture().get("batch1024_sample/jacobi/rtol1e-12")
    if not rec or len(systems) != 1024 or batch_cpu_sample(systems) != rec["indices"]:
        return None
    import scipy.sparse as sp
    errs, trs = [], []
    for i in rec["indices"]:
        s, r, ref = systems[i], results[i], rec["systems"][str(i)]
        if (s.n, s.nnz) != (ref["n"], ref["nnz"]):
            return None
        e = P.probe_error(P.solution_probe(r.x), ref["probe"])
        errs.append(max(e["proj"], e["sample"]))
        A = sp.csr_matrix((s.val, s.col, s.rowptr), shape=(s.n, s.n))
        trs.append(float(np.linalg.norm(s.b - A @ r.x) / np.linalg.norm(s.b)))
    return {"worst": float(max(errs)), "median": float(np.median(errs)), "systems": len(errs),
            "true_rel_residual_worst": float(max(trs)),
            "oracle": "HiFlow3 lmp CG, FP64 Jacobi-PCG to rel. 1e-12, on the stratified CPU sample "
                      "(tests/golden/reference_fullsize_solutions.json)",
            "estimate": "||x - x_ref|| / ||x_ref|| from 64 Rademacher projections and 2,048 sampled entries"}


def _pinned(a, torch):
    t = torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
    return t, t.numpy()


def run_batch(args, rank, local_rank, world, torch, dist, barrier):
    from ba_b200 import lmp
    from ba_b200.batch import Batch

    plat = lmp.Platform(local_rank)
    stream = work_stream(torch)
    plat.set_stream(stream.cuda_stream)
    all_systems = make_batch_systems(args.count, 0 if args.split else rank)
    systems = all_systems
    if args.split and world > 1:
        # one batch shared by all ranks, cut by cost (nnz): no data-path exchange
        parts = D.partition_by_cost([t.nnz for t in all_systems], world)
        systems = [all_systems[i] for i in parts[rank]]
    keep, host = [], []
    for s in systems:
        arrs = [_pinned(a, torch) for a in (s.rowptr, s.col, s.val, s.b)]
        keep.append([t for t, _ in arrs])
        host.append([a for _, a in arrs])
    cap = len(systems)
    inner_rtol = args.inner_rtol if args.inner_rtol is not None else BATCH_INNER
    kw = dict(mixed=True, precond=True, rtol=BATCH_RTOL, atol=0.0, dtol=1e8, inner_rtol=inner_rtol, max_outer=60,
              platform=plat)
    B = Batch(cap, **kw)
    for h in host:
        B.add(*h)
    item_rows, _ = B.tune()

    def step():
        B.restart()
        return B.solve(CHUNK)

    for _ in range(args.warmup):
        passes = step()
    clocks = ClockSampler(local_rank)
    barrier()
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    passes_tot = 0
    for _ in range(args.steps):
        passes_tot += step()
    e1.record(stream)
    e1.synchronize()
    barrier()
    clk = clocks.stop()
    ms_max = D.max_over_ranks(e0.elapsed_time(e1))
    solved_per_step = len(all_systems) if args.split else world * len(systems)
    value = args.steps * solved_per_step / (ms_max / 1e3)

    # per-system results of the last step: states, latency inside the step, accuracy
    res = [B.result(k, with_x=True) for k in range(len(systems))]
    solve_bytes = batch_solver_bytes(systems, res)
    ok = sum(1 for r in res if r.solver_state == 0)
    lat = np.array([r.device_us for r in res]) / 1e3
    iters = np.array([r.iters for r in res])
    outer = np.array([r.outer for r in res])
    import scipy.sparse as sp
    worst = 0.0
    for s, r in zip(systems[::64], res[::64]):
        A = sp.csr_matrix((s.val, s.col, s.rowptr), shape=(s.n, s.n))
        worst = max(worst, float(np.linalg.norm(s.b - A @ r.x) / np.linalg.norm(s.b)))

    err_oracle = batch_error_vs_cpu_oracle(systems, res) if rank == 0 else None

    # FP64 comparators on the same machinery and batch: the plain FP64 GPU CG
    # (SolveNoPrecond recurrence, the north-star denominator) and FP64
    # Jacobi-PCG (what the mixed precision itself buys)
    def fp64_batch(precond):
        Pn = Batch(cap, mixed=False, precond=precond, rtol=BATCH_RTOL, atol=0.0, dtol=1e8, inner_maxits=1000000,
                   platform=plat)
        for h in host:
            Pn.add(*h)
        Pn.tune()
        Pn.restart()
        Pn.solve(CHUNK)
        barrier()
        k_plain = max(2, args.steps // 2)
        c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        c0.record(stream)
        for _ in range(k_plain):
            Pn.restart()
            Pn.solve(CHUNK)
        c1.record(stream)
        c1.synchronize()
        rate = len(systems) * k_plain / (c0.elapsed_time(c1) / 1e3)
        its = np.array([Pn.result(k, with_x=False).iters for k in range(len(systems))])
        Pn.close()
        return rate, its

    plain_value, plain_iters = fp64_batch(False)
    pcg_value, pcg_iters = fp64_batch(True)

    # end to end through the public API: upload every system from pinned host
    # memory, solve, download every solution, each step
    E = Batch(cap, **kw)
    E.set_items(*B.items(), adaptive=False)  # the schedule tuned on the full batch
    xs = [torch.empty(s.n, dtype=torch.float64).pin_memory().numpy() for s in systems]
    h2d = int(sum(h[0].nbytes + h[1].nbytes + h[2].nbytes + h[3].nbytes for h in host))
    d2h = int(sum(x.nbytes for x in xs))
    # the systems go up in chunks, largest first, each chunk's upload overlapping
    # the passes already running on the chunks before it (adds run on the
    # batch's transfer stream, launches are asynchronous)
    order = sorted(range(len(systems)), key=lambda k: -systems[k].n)
    chunks, at = [], 0
    for size in E2E_CHUNKS:
        chunks.append(order[at:at + size])
        at += size
    if at < len(order):
        chunks.append(order[at:])
    chunks = [c for c in chunks if c]

    slot_of = {}

    def e2e_step():
        if slot_of:
            E.remove_many(list(slot_of.values()))
        slot_of.clear()
        for ch in chunks:
            sls = E.add_many([host[k] for k in ch])
            for k, sl in zip(ch, sls):
                slot_of[k] = sl
            # each solution is copied out as soon as its system finishes
            E.set_outputs(sls, [xs[k] for k in ch])
            E.launch(E2E_LAUNCH_PASSES)
        E.solve(CHUNK)
        E.results([slot_of[k] for k in range(len(systems))], out=xs)

    e2e_step()
    barrier()
    h0, h1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    k_e2e = max(2, args.steps // 2)
    h0.record(stream)
    for _ in range(k_e2e):
        e2e_step()
    h1.record(stream)
    h1.synchronize()
    e2e_value = k_e2e * solved_per_step / (D.max_over_ranks(h0.elapsed_time(h1)) / 1e3)
    E.close()

    # roofline of the dominant kernel: K1 of the inner solve (batched FP32
    # sliced-ELL SpMV fused with p.Ap), timed launch by launch with CUDA
    # events on the solve stream over a full inner pass of every system
    B.profile_pass(5)  # warms the GPU up after the host-bound e2e loop
    pass_ms, pass_bytes = B.profile_pass(5)
    spmv_ms, spmv_bytes_alg = pass_ms[0], pass_bytes[0]
    peak, peak_kind = measured_peak_gbs()
    achieved = spmv_bytes_alg / (spmv_ms / 1e3) / 1e9
    kernels = {name: {"ms": t, "algorithmic_bytes": b, "gbs": b / (t / 1e3) / 1e9}
               for name, t, b in zip(("K1_spmv_pAp", "K2_update", "K3_direction"), pass_ms, pass_bytes)}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        import oracle
        if oracle.ref_available():
            nthreads = os.cpu_count() or 1
            pick = batch_cpu_sample(systems)
            cnt, sec = ref_batch_sample(systems, pick, nthreads)
            cpu = {"value": cnt / sec, "unit": "solves/s", "cores": nthreads, "kind": "reference",
                   "sample": batch_cpu_sample_text(args, pick, nthreads)}
    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "strong" if args.split else "weak", "vs_baseline": None, "dtype": "f32+f64",
            "data": "synthetic",
            "config": batch_config(args, all_systems),
            "details": {
                "parallelism": (f"split x{world}: one batch partitioned over the ranks by nnz (greedy, largest "
                                f"first); rank 0 solved {len(systems)} systems") if args.split
                               else f"replicas x{world}: every rank solves its own seeded batch",
                "precision": f"FP32 Jacobi-PCG inner solves (FP32 matrix values and vectors, compensated FP32 "
                             f"dots) inside FP64 refinement: the FP64 residual replaces the inner one every "
                             f"{inner_rtol:g}x reduction, the search direction is kept",
                "spmv_schedule": ("sliced ELL, 32 rows per slice, one row per lane; values only (columns = row + the "
                                  "system's 9 stencil offsets), p window staged in shared memory"),
                "p50_latency_ms": float(np.percentile(lat, 50)), "p99_latency_ms": float(np.percentile(lat, 99)),
                "latency": "per-system device time from its first residual to its finish inside the step",
                "converged": f"{ok}/{len(systems)}", "worst_true_rel_residual_sampled": worst,
                "error_vs_cpu_oracle": err_oracle,
                "inner_iters_mean": float(iters.mean()), "inner_iters_max": int(iters.max()),
                "refinement_passes_max": int(outer.max()), "device_loop_passes_per_step": passes_tot / args.steps,
                "solver_algorithmic_bytes_per_step": solve_bytes,
                "solver_effective_gbs": solve_bytes / (ms_max / args.steps / 1e3) / 1e9,
                "plain_fp64_cg": {"value": plain_value, "unit": "solves/s",
                                  "iters_mean": float(plain_iters.mean()), "iters_max": int(plain_iters.max()),
                                  "speedup_of_mixed_pcg": value / world / plain_value},
                "fp64_jacobi_pcg": {"value": pcg_value, "unit": "solves/s",
                                    "iters_mean": float(pcg_iters.mean()), "iters_max": int(pcg_iters.max()),
                                    "speedup_of_mixed_pcg": value / world / pcg_value}},
            "clocks": clk,
            "e2e": {"value": e2e_value, "unit": "solves/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": args.steps + 3 * passes_tot + (passes_tot + CHUNK - 1) // CHUNK,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": profile_traffic("batch1024/f32/spmv"), "peak_source": peak_kind,
                         "kernel": "batch_spmv_kernel<float> (K1: sliced-ELL SpMV + p.Ap) over an inner pass of "
                                   "all 1024 systems",
                         "algorithmic_bytes": spmv_bytes_alg, "kernel_ms": spmv_ms, "pass_kernels": kernels,
                         "item_rows": {"spmv": item_rows[0], "update": item_rows[1], "direction": item_rows[2]},
                         **dram_rate(profile_traffic("batch1024/f32/spmv"), spmv_ms, peak)},
            "cpu_baseline": cpu,
        }
        print(json.dumps(out))
    B.close()


# mixed batch: an inner pass ends at this reduction of its residual, which the
# FP64 residual then replaces (direction kept); 0.1 was the fastest of
# 0.03 / 0.1 / 0.3 on the 1,024-system batch
BATCH_INNER = 0.1

# e2e: upload chunks (largest systems first: the first, small chunk starts the
# slowest systems after a few ms) and passes per overlapping launch
E2E_CHUNKS = (8, 24, 64, 160, 256)
E2E_LAUNCH_PASSES = 128


# ----------------------------------------------------------------- serve workload
SERVE_CAPACITY = 256


SERVE_STREAM = 20000  # requests in the seeded served stream


def serve_requests(count: int, rate: float, hi_dofs: float, rank: int, offset: int = 0):
    """Requests offset..offset+count-1 of the seeded served stream (2D/3D Q1
    diffusion, DOFs log-uniform in [1e3, hi_dofs], sigma U[0.5, 2])."""
    from ba_b200 import problems as P
    return P.serve_stream(offset + count, rate=rate, hi_dofs=hi_dofs, seed=D.rank_seed(P.SEED_SERVE, rank))[offset:]


def serve_sample(count: int, hi_dofs: float, rank: int, part: int = 0, rate: float = 1.0):
    """A size-stratified sample of `count` requests of the seeded 20,000-request
    stream (part 0 and part 1 are disjoint: the sample is drawn from the even
    or the odd requests), re-timed as Poisson arrivals at `rate` per second."""
    from ba_b200 import problems as P
    stream = P.serve_stream(SERVE_STREAM, rate=1.0, hi_dofs=hi_dofs, seed=D.rank_seed(P.SEED_SERVE, rank))
    pool = stream[part::2]
    pick = P.stratified_sample([rq["dofs"] for rq in pool], count)
    gaps = -np.log1p(-P.uniform01(P.SEED_SERVE + 77 + part, len(pick), stream=31)) / rate
    t = np.cumsum(gaps) - gaps[0]
    return [dict(pool[i], t=float(ti)) for i, ti in zip(pick, t)]


def serve_config(args, extra=None):
    cfg = {"workload": f"served: Poisson-arrival stream of 2D/3D Q1 diffusion solves, DOFs logU[1e3,{args.hi_dofs:.0e}], "
                       f"lognormal kappa sigma~U[0.5,2], rel. residual 1e-8",
           "requests_per_step": args.requests,
           "requests_note": "a size-stratified sample of the seeded 20,000-request stream (the middle request of "
                            "each of steps x requests_per_step equal-count DOF strata of its even requests); "
                            "each is assembled on the device from (dim, cells, seed, sigma) at admission",
           "l2": "inputs larger than L2 (each step's matrices total several GB)"}
    if extra:
        cfg.update(extra)
    return cfg


def ref_serve_sample(reqs, nthreads: int, max_dofs: float, budget_s: float):
    """The reference's CPU CG (FP64 Jacobi-PCG, OPENMP SpMV) to 1e-8 on the
    stream's requests of at most max_dofs DOFs, in order, until budget_s of
    solve time is spent; returns (solves, seconds)."""
    import oracle
    from ba_b200 import problems as P
    total, cnt = 0.0, 0
    for rq in reqs:
        if rq["dofs"] > max_dofs:
            continue
        s = P.q1_system(rq["dim"], rq["cells"], rq["seed"], rq["sigma"])
        ref = oracle.RefSystem(s.rowptr, s.col, s.val, impl=oracle.IMPL_OPENMP, nthreads=nthreads)
        _, sec = ref.cg(s.b, maxits=100000, atol=0.0, rtol=BATCH_RTOL, dtol=1e8, precond=True)
        ref.close()
        total += sec
        cnt += 1
        if total >= budget_s:
            break
    return cnt, total


def run_reference_serve(args, rank):
    import oracle
    if not oracle.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built (reference sources absent)"}))
        return
    nthreads = os.cpu_count() or 1
    reqs = serve_sample(args.steps * args.requests, args.hi_dofs, 0, part=0)
    rates, secs = [], []
    for step in range(args.warmup + args.steps):
        cnt, sec = ref_serve_sample(reqs, nthreads, 1e5, 3.0)
        if step >= args.warmup:
            rates.append(cnt / sec)
            secs.append(sec)
    value = statistics.median(rates)
    sample = (f"per step, the requests of at most 1e5 DOFs of the timed stratified sample, in order, solved to "
              f"1e-8 by HiFlow3 lmp CG (FP64 Jacobi-PCG, OPENMP SpMV, {nthreads} threads) until 3 s of solve "
              f"time; larger requests are skipped, which favours the reference")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * statistics.median(secs),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": serve_config(args),
        "details": {"parallelism": f"cpu openmp x{nthreads}", "step": sample},
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": nthreads, "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))

def _serve_stream(S, reqs, paced: bool, timeout: float = 1800.0):
    """Submits reqs (paced by their arrival times, or all at once), waits for
    all of them, fetches every solution; returns the results."""
    t0 = time.monotonic()
    ids = []
    for rq in reqs:
        if paced:
            d = t0 + rq["t"] - time.monotonic()
            if d > 0:
                time.sleep(d)
        ids.append(S.submit_q1(rq["dim"], rq["cells"], rq["seed"], rq["sigma"]))
    S.drain(timeout)
    out = []
    for rid in ids:
        r, lat = S.poll(rid, with_x=True)
        out.append((r, lat))
        S.release(rid)
    return out


def run_serve(args, rank, local_rank, world, torch, dist, barrier):
    from ba_b200 import lmp
    from ba_b200.server import Server

    plat = lmp.Platform(local_rank)
    stream = work_stream(torch)
    plat.set_stream(stream.cuda_stream)
    inner_rtol = args.inner_rtol if args.inner_rtol is not None else BATCH_INNER
    kw = dict(rtol=BATCH_RTOL, atol=0.0, dtol=1e8, inner_rtol=inner_rtol, max_outer=60, chunk_passes=CHUNK,
              platform=plat)
    R = args.requests
    split = args.split and world > 1

    def req_cost(rq):  # a request's work: its matrix nonzeros (9 or 27 per row)
        return rq["dofs"] * (9 if rq["dim"] == 2 else 27)

    def my_share(reqs, drain_rate):
        # every rank routes the same global stream the same way and keeps its part
        return D.stream_share(reqs, world, rank, drain_rate, req_cost)

    if split:
        all_timed = serve_sample(world * args.steps * R, args.hi_dofs, 0, part=0)
        timed = my_share(all_timed, 0.0)
    else:
        timed = serve_sample(args.steps * R, args.hi_dofs, rank, part=0)
    warm = serve_requests(args.warmup * 4, 1.0, 2e4, rank, offset=50000)
    S = Server(SERVE_CAPACITY, mixed=True, precond=True, **kw)
    for w in range(args.warmup):
        _serve_stream(S, warm[4 * w:4 * w + 4], paced=False)
    clocks = ClockSampler(local_rank)
    barrier()
    clocks.start()
    S.reset_stats()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    # the whole timed stream arrives at once: the server admits it as slots
    # and memory allow, so the measure is saturated throughput with one tail
    results = _serve_stream(S, timed, paced=False)
    e1.record(stream)
    e1.synchronize()
    barrier()
    clk = clocks.stop()
    st_sat = S.stats()
    ms_max = D.max_over_ranks(e0.elapsed_time(e1))
    value = world * args.steps * R / (ms_max / 1e3)
    # work a GPU drains per second at saturation (the split streams' routing)
    drain = (sum(req_cost(rq) for rq in all_timed) / world if split else 0.0) / (ms_max / 1e3)
    ok = sum(1 for r, _ in results if r.solver_state == 0)
    d2h = int(sum(r.x.nbytes for r, _ in results)) // args.steps
    h2d = 4 * 8 * R  # request descriptors per step: dim, cells, seed, sigma

    # latency under a Poisson stream at a fraction of the measured throughput
    rate = max(args.load * value / world, 1e-3)
    if split:
        lat_reqs = my_share(serve_sample(world * args.latency_requests, args.hi_dofs, 0, part=1, rate=world * rate),
                            drain)
    else:
        lat_reqs = serve_sample(args.latency_requests, args.hi_dofs, rank, part=1, rate=rate)
    S.reset_stats()
    lat_res = _serve_stream(S, lat_reqs, paced=True)
    st_lat = S.stats()
    lat_ok = sum(1 for r, _ in lat_res if r.solver_state == 0)
    worst_rel = max(r.res_rel for r, _ in results + lat_res)
    full = None
    if args.full_stream:
        # the whole seeded stream, Poisson arrivals at the same fraction of the
        # measured throughput; only the result records are kept
        if split:
            full_reqs = my_share(serve_requests(args.stream_count, world * rate, args.hi_dofs, 0), drain)
        else:
            full_reqs = serve_requests(args.stream_count, rate, args.hi_dofs, rank)
        S.reset_stats()
        f0 = time.monotonic()
        pending, full_rs = [], []

        def harvest():
            # finished requests give up their stored solutions at once, so the
            # host holds only what is in flight
            keep = []
            for rid in pending:
                got = S.poll(rid, with_x=False)
                if got is None:
                    keep.append(rid)
                else:
                    full_rs.append(got[0])
                    S.release(rid)
            pending[:] = keep

        for k, rq in enumerate(full_reqs):
            d = f0 + rq["t"] - time.monotonic()
            if d > 0:
                time.sleep(d)
            pending.append(S.submit_q1(rq["dim"], rq["cells"], rq["seed"], rq["sigma"]))
            if k % 256 == 255:
                harvest()
        S.drain(7200.0)
        harvest()
        st_full = S.stats()
        full = {"requests": len(full_reqs), "arrival_rate_per_s": rate, "wall_s": time.monotonic() - f0,
                "solves_per_s": st_full["solves_per_s"], "p50_ms": st_full["p50_ms"], "p99_ms": st_full["p99_ms"],
                "mean_ms": st_full["mean_ms"], "max_ms": st_full["max_ms"],
                "converged": f"{sum(1 for r in full_rs if r.solver_state == 0)}/{len(full_rs)}",
                "worst_rel_residual": max(r.res_rel for r in full_rs),
                "dofs_mean": float(np.mean([rq["dofs"] for rq in full_reqs])),
                "dofs_total": int(sum(rq["dofs"] for rq in full_reqs)),
                "hbm_peak_bytes": st_full["hbm_peak"], "launches": st_full["launches"],
                "device_passes": st_full["passes"]}
    S.close()

    # plain FP64 GPU CG (unpreconditioned recurrence) on exactly the timed requests, served the same way
    Pn = Server(SERVE_CAPACITY, mixed=False, precond=False, inner_maxits=1000000, **{
        k: v for k, v in kw.items() if k not in ("inner_rtol", "max_outer")})
    _serve_stream(Pn, warm[:4], paced=False)
    barrier()
    c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    c0.record(stream)
    plain_res = _serve_stream(Pn, timed, paced=False)
    c1.record(stream)
    c1.synchronize()
    plain_value = len(timed) / (c0.elapsed_time(c1) / 1e3)
    plain_ok = sum(1 for r, _ in plain_res if r.solver_state == 0)
    plain_iters_max = max(r.iters for r, _ in plain_res)
    Pn.close()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        import oracle
        if oracle.ref_available():
            nthreads = os.cpu_count() or 1
            cnt, sec = ref_serve_sample(timed, nthreads, 1e5, 15.0)
            cpu = {"value": cnt / sec, "unit": "solves/s", "cores": nthreads, "kind": "reference",
                   "sample": f"{cnt} requests of at most 1e5 DOFs from the timed stream, solved to 1e-8 by "
                             f"HiFlow3 lmp CG (FP64 Jacobi-PCG, OPENMP SpMV, {nthreads} threads); larger "
                             f"requests skipped, which favours the reference"}
    if rank == 0:
        dofs = [rq["dofs"] for rq in timed]
        print(json.dumps({
            "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
            "config": serve_config(args),
            "details": {
                "parallelism": (f"split x{world}: one request stream ({world}x the requests) routed over the "
                                f"ranks, join-shortest-queue by outstanding nonzeros" if split
                                else f"replicas x{world}"),
                "server": f"FP32 Jacobi-PCG inner solves in FP64 refinement (residual replaced every "
                          f"{inner_rtol:g}x, direction kept), admitted by free HBM into {SERVE_CAPACITY} slots, "
                          f"continuous batching",
                "throughput_stream": "all steps x requests_per_step requests submitted at once; ms_per_step = "
                                     "time to drain / steps",
                "converged": f"{ok}/{len(results)}", "dofs_mean": float(np.mean(dofs)), "dofs_max": int(max(dofs)),
                "worst_rel_residual": worst_rel,
                "hbm_peak_bytes": st_sat["hbm_peak"], "hbm_budget_bytes": st_sat["hbm_budget"],
                "launches": st_sat["launches"], "device_passes": st_sat["passes"],
                "latency_stream": {"requests": len(lat_reqs), "arrival_rate_per_s": rate,
                                   "p50_ms": st_lat["p50_ms"], "p99_ms": st_lat["p99_ms"],
                                   "mean_ms": st_lat["mean_ms"], "max_ms": st_lat["max_ms"],
                                   "solves_per_s": st_lat["solves_per_s"], "converged": f"{lat_ok}/{len(lat_res)}",
                                   "latency": "submission to solution on the host"},
                "burst_latency_p50_ms": st_sat["p50_ms"], "burst_latency_p99_ms": st_sat["p99_ms"],
                "plain_fp64_cg": {"value": plain_value, "unit": "solves/s", "requests": len(timed),
                                  "converged": f"{plain_ok}/{len(timed)}", "iters_max": plain_iters_max,
                                  "speedup_of_mixed_pcg": value / world / plain_value},
                "full_stream": full},
            "clocks": clk,
            "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "note": "the timed region is end to end: submission of request descriptors, device assembly, "
                            "solve, solution copied to host memory"},
            # 3 kernels per device pass; per request: coefficient, assembly and slot setup kernels
            "gpu_launches": int(3 * st_sat["passes"] + 3 * args.steps * R),
            "roofline": None,
            "cpu_baseline": cpu}))


# ----------------------------------------------------------------- poisson3d workload
def run_reference_poisson3d(args, rank):
    import oracle
    from ba_b200 import problems as P
    if not oracle.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built (reference sources absent)"}))
        return
    s = P.poisson_3d(args.cells)
    counts = json.load(open(COUNTS)) if os.path.exists(COUNTS) else {}
    full_iters = counts.get(f"poisson3d_{args.cells}/jacobi/rtol1e-10", {}).get("iters", 20)
    nthreads = os.cpu_count() or 1
    ref = oracle.RefSystem(s.rowptr, s.col, s.val, impl=oracle.IMPL_OPENMP, nthreads=nthreads)
    sample_iters = 20
    per_iter = []
    for step in range(args.warmup + args.steps):
        r, sec = ref.cg(s.b, maxits=sample_iters, atol=0.0, rtol=1e-10, dtol=1e8, precond=True)
        if step >= args.warmup:
            per_iter.append(sec / max(r.iters, 1))
    value = 1.0 / (statistics.median(per_iter) * full_iters)
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 / value, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": poisson3d_config(args, s),
        "details": {"parallelism": f"cpu openmp x{nthreads}", "iters_per_solve": full_iters,
                    "step": f"{sample_iters} of {full_iters} iterations of one solve, scaled to a full solve"},
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": nthreads, "kind": "reference",
                         "sample": f"{sample_iters} of {full_iters} iterations of one solve per step, scaled"},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))


def poisson3d_config(args, s):
    return {"workload": f"fp64 jacobi-pcg 3d q1 poisson {args.cells}^3 cells, rel 1e-10", "n": s.n, "nnz": s.nnz,
            "l2": "inputs larger than L2 (matrix 685 MB streamed per iteration)"}


def fullsize_check(name, rtol_key, x, iters):
    """Iteration count and error of a device solution against the reference's
    recorded run of the same workload (None if not recorded)."""
    from ba_b200 import problems as P
    rec = fullsize_fixture().get(f"{name}/jacobi/{rtol_key}")
    if not rec or rec["n"] != x.shape[0]:
        return None
    e = P.probe_error(P.solution_probe(x), rec["probe"])
    return {"reference_iters": rec["iters"], "iters": iters, "error": max(e["proj"], e["sample"]),
            "reference": f"HiFlow3 lmp CG (NAIVE, FP64 Jacobi-PCG) to {rtol_key[4:]}, recorded fingerprints",
            "estimate": "||x - x_ref|| / ||x_ref|| from 64 Rademacher projections and 2,048 sampled entries"}


def run_poisson3d(args, rank, local_rank, world, torch, dist, barrier):
    import ctypes as C

    from ba_b200 import lmp
    from ba_b200 import problems as P
    from ba_b200._lib import FORMAT_NAMES, load

    plat = lmp.Platform(local_rank)
    stream = work_stream(torch)
    plat.set_stream(stream.cuda_stream)
    s = P.poisson_3d(args.cells)
    n, nnz = s.n, s.nnz
    A = lmp.B200_CSR_lMatrix(s.rowptr, s.col, s.val, platform=plat)
    fmt, prm, _ = A.tune()
    b = lmp.B200_lVector.from_numpy(s.b, platform=plat)
    x = lmp.B200_lVector(n, platform=plat)
    solver = lmp.setup_CG_solver(maxits=20000, atol=0.0, rtol=1e-10, dtol=1e8, use_precond=True)
    solver.SetupOperator(A)
    plain = lmp.setup_CG_solver(maxits=20000, atol=0.0, rtol=1e-10, dtol=1e8, use_precond=False)
    plain.SetupOperator(A)

    def step(sv):
        x.Zeros()
        assert sv.Solve(b, x) == lmp.kSolverSuccess
        return sv.iter()

    for _ in range(args.warmup):
        step(solver)
    iters = solver.iter()
    clocks = ClockSampler(local_rank)
    barrier()
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step(solver)
    e1.record(stream)
    e1.synchronize()
    barrier()
    clk = clocks.stop()
    ms_max = D.max_over_ranks(e0.elapsed_time(e1))
    value = world * args.steps / (ms_max / 1e3)
    parity = fullsize_check(f"poisson3d_{args.cells}", "rtol1e-10", x.numpy(), iters) if rank == 0 else None
    step(plain)
    c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    k_plain = max(2, args.steps // 2)
    c0.record(stream)
    for _ in range(k_plain):
        step(plain)
    c1.record(stream)
    c1.synchronize()
    plain_value = k_plain / (c0.elapsed_time(c1) / 1e3)
    lib = load()
    bh = torch.from_numpy(s.b).pin_memory()
    xh = torch.empty(n, dtype=torch.float64).pin_memory()
    barrier()
    h0, h1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    h0.record(stream)
    for _ in range(args.steps):
        lib.b200la_vec_upload(b.handle, C.c_void_p(bh.data_ptr()), n)
        step(solver)
        lib.b200la_vec_download(x.handle, C.c_void_p(xh.data_ptr()), n)
    h1.record(stream)
    h1.synchronize()
    e2e_value = D.aggregate_rate(args.steps, world, D.max_over_ranks(h0.elapsed_time(h1)))
    ms3 = (C.c_double * 3)()
    for _ in range(2):  # the first call warms the GPU up after the host-bound e2e loop
        x.Zeros()
        lib.b200la_cg_profile(solver._solver, b.handle, x.handle, 20, ms3)
    bytes_spmv = spmv_bytes(n, nnz, 8)
    peak, peak_kind = measured_peak_gbs()
    achieved = bytes_spmv / (ms3[0] / 1e3) / 1e9
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        import oracle
        if oracle.ref_available():
            counts = json.load(open(COUNTS)) if os.path.exists(COUNTS) else {}
            full = counts.get(f"poisson3d_{args.cells}/jacobi/rtol1e-10", {}).get("iters", iters)
            nthreads = os.cpu_count() or 1
            ref = oracle.RefSystem(s.rowptr, s.col, s.val, impl=oracle.IMPL_OPENMP, nthreads=nthreads)
            r, sec = ref.cg(s.b, maxits=20, atol=0.0, rtol=1e-10, dtol=1e8)
            cpu = {"value": 1.0 / (sec / max(r.iters, 1) * full), "unit": "solves/s", "cores": nthreads,
                   "kind": "reference", "sample": f"20 of {full} iterations of one solve (HiFlow3 lmp OPENMP "
                                                  f"SpMV, {nthreads} threads), scaled to a full solve"}
    if rank == 0:
        print(json.dumps({
            "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": poisson3d_config(args, s),
            "details": {"iters_per_solve": iters, "parallelism": f"replicas x{world}",
                        "spmv_schedule": FORMAT_NAMES[fmt] + f"/{prm}",
                        "parity_vs_reference": parity,
                        "plain_fp64_cg": {"value": plain_value, "unit": "solves/s", "iters_per_solve": plain.iter()}},
            "clocks": clk,
            "e2e": {"value": e2e_value, "unit": "solves/s", "h2d_bytes_per_step": n * 8, "d2h_bytes_per_step": n * 8},
            "gpu_launches": args.steps * (1 + 3 * iters),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": profile_traffic(f"poisson3d_{args.cells}/f64/spmv"), "peak_source": peak_kind,
                         "kernel": "cg_spmv_kernel (SpMV fused with p.Ap)", "algorithmic_bytes": bytes_spmv,
                         "kernel_ms": {"spmv_dot": ms3[0], "update": ms3[1], "direction": ms3[2]},
                         **dram_rate(profile_traffic(f"poisson3d_{args.cells}/f64/spmv"), ms3[0], peak)},
            "cpu_baseline": cpu}))


# ----------------------------------------------------------------- varcoef3d workload
def varcoef3d_config(args, s):
    return {"workload": f"3d q1 lognormal sigma=2 diffusion {args.cells}^3 cells, rel 1e-10", "n": s.n,
            "nnz": s.nnz, "l2": "inputs larger than L2 (FP32 matrix 456 MB + FP64 matrix 685 MB)"}


def varcoef3d_fp64_iters(cells):
    """The reference's FP64 Jacobi-PCG iteration count on the varcoef3d system (its
    recorded run), else None."""
    rec = fullsize_fixture().get(f"varcoef3d_{cells}/jacobi/rtol1e-10")
    return rec["iters"] if rec else None


def run_reference_varcoef3d(args, rank):
    import oracle
    from ba_b200 import problems as P
    if not oracle.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built (reference sources absent)"}))
        return
    s = P.varcoef_3d(args.cells, sigma=2.0)
    full_iters = varcoef3d_fp64_iters(args.cells)
    nthreads = os.cpu_count() or 1
    ref = oracle.RefSystem(s.rowptr, s.col, s.val, impl=oracle.IMPL_OPENMP, nthreads=nthreads)
    sample_iters = 20
    per_iter = []
    for step in range(args.warmup + args.steps):
        r, sec = ref.cg(s.b, maxits=sample_iters, atol=0.0, rtol=1e-10, dtol=1e8, precond=True)
        if step >= args.warmup:
            per_iter.append(sec / max(r.iters, 1))
    if full_iters is None:  # not recorded for this size: run the whole solve once
        r, _ = ref.cg(s.b, maxits=100000, atol=0.0, rtol=1e-10, dtol=1e8, precond=True)
        full_iters = r.iters
    value = 1.0 / (statistics.median(per_iter) * full_iters)
    step_text = (f"{sample_iters} iterations of FP64 Jacobi-PCG per step (HiFlow3 lmp OPENMP SpMV, {nthreads} "
                 f"threads), scaled by the reference's {full_iters} iterations per solve")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * statistics.median(per_iter) * sample_iters, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": varcoef3d_config(args, s),
        "details": {"parallelism": f"cpu openmp x{nthreads}", "step": step_text,
                    "full_solve_ms_extrapolated": 1e3 / value},
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": nthreads, "kind": "reference",
                         "sample": step_text},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))


# varcoef3d mixed precision: the FP64 residual replaces the inner one every
# VARCOEF_INNER reduction (direction kept)
VARCOEF_INNER = 0.1


def run_varcoef3d(args, rank, local_rank, world, torch, dist, barrier):
    import ctypes as C

    from ba_b200 import lmp
    from ba_b200 import problems as P
    from ba_b200._lib import load

    plat = lmp.Platform(local_rank)
    stream = work_stream(torch)
    plat.set_stream(stream.cuda_stream)
    s = P.varcoef_3d(args.cells, sigma=2.0)
    n, nnz = s.n, s.nnz
    A = lmp.B200_CSR_lMatrix(s.rowptr, s.col, s.val, platform=plat)
    A.tune()
    b = lmp.B200_lVector.from_numpy(s.b, platform=plat)
    x = lmp.B200_lVector(n, platform=plat)
    inner_rtol = args.inner_rtol if args.inner_rtol is not None else VARCOEF_INNER
    m = lmp.MPIR()
    m.SetupOperator(A)
    m.SetMpirParameters(0, 60, 0.0, 1e-10, 1e6)
    m.SetLowPrecErrCorSolverParameters(200000, 0.0, inner_rtol, 1e30)

    def mp_step(solver=m):
        x.Zeros()
        st = solver.Solve(b, x)
        assert st == lmp.kSolverSuccess, (solver.state_, solver.res_rel_)

    for _ in range(args.warmup):
        mp_step()
    clocks = ClockSampler(local_rank)
    barrier()
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        mp_step()
    e1.record(stream)
    e1.synchronize()
    barrier()
    clk = clocks.stop()
    ms_max = D.max_over_ranks(e0.elapsed_time(e1))
    value = world * args.steps / (ms_max / 1e3)
    x_mp = x.numpy().copy()
    outer, inner = m.outer_, m.iter()

    # FP64 comparators on the same matrix: Jacobi-PCG and plain CG
    def fp64_rate(precond, rtol, reps):
        sv = lmp.setup_CG_solver(maxits=500000, atol=0.0, rtol=rtol, dtol=1e8, use_precond=precond)
        sv.SetupOperator(A)
        x.Zeros()
        sv.Solve(b, x)
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        for _ in range(reps):
            x.Zeros()
            st = sv.Solve(b, x)
        f1.record(stream)
        f1.synchronize()
        return reps / (f0.elapsed_time(f1) / 1e3), sv.iter(), st

    pcg_value, pcg_iters, _ = fp64_rate(True, 1e-10, 2)
    x_pcg = x.numpy().copy()
    plain_value, plain_iters, plain_state = fp64_rate(False, 1e-10, 1)
    # MPIR's own form for comparison: the FP32 inner solve restarted every pass
    mr = lmp.MPIR()
    mr.SetupOperator(A)
    mr.SetInnerRestart(True)
    mr.SetMpirParameters(0, 60, 0.0, 1e-10, 1e6)
    mr.SetLowPrecErrCorSolverParameters(200000, 0.0, 1e-5, 1e30)
    mp_step(mr)
    r0, r1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    r0.record(stream)
    mp_step(mr)
    r1.record(stream)
    r1.synchronize()
    restart_value, restart_iters, restart_passes = 1e3 / r0.elapsed_time(r1), mr.iter(), mr.outer_
    mr._release()
    # errors against the FP64 CPU CG oracle: the reference's own CG to 1e-13
    # (recorded fingerprints); else a device FP64 Jacobi-PCG to 1e-13
    from ba_b200 import problems as P_
    rec13 = fullsize_fixture().get(f"varcoef3d_{args.cells}/jacobi/rtol1e-13")
    if rec13 and rec13["n"] == n:
        probe13 = rec13["probe"]
        err_ref = "HiFlow3 lmp CG (NAIVE, FP64 Jacobi-PCG) to 1e-13, recorded fingerprints"
    else:
        refs = lmp.setup_CG_solver(maxits=500000, atol=0.0, rtol=1e-13, dtol=1e8, use_precond=True)
        refs.SetupOperator(A)
        x.Zeros()
        refs.Solve(b, x)
        probe13 = P_.solution_probe(x.numpy())
        err_ref = "device FP64 Jacobi-PCG to 1e-13 (no recorded reference run at this size)"

    def err_of(xv):
        e = P_.probe_error(P_.solution_probe(xv), probe13)
        return max(e["proj"], e["sample"])

    err = err_of(x_mp)
    err_pcg = err_of(x_pcg)
    import scipy.sparse as sp
    Ah = sp.csr_matrix((s.val, s.col, s.rowptr), shape=(n, n))
    true_rel = float(np.linalg.norm(s.b - Ah @ x_mp) / np.linalg.norm(s.b))

    # e2e through the public API: RHS up from pinned host memory, solve, solution down
    lib = load()
    bh = torch.from_numpy(s.b).pin_memory()
    xh = torch.empty(n, dtype=torch.float64).pin_memory()
    barrier()
    h0, h1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    h0.record(stream)
    for _ in range(args.steps):
        lib.b200la_vec_upload(b.handle, C.c_void_p(bh.data_ptr()), n)
        mp_step()
        lib.b200la_vec_download(x.handle, C.c_void_p(xh.data_ptr()), n)
    h1.record(stream)
    h1.synchronize()
    e2e_value = D.aggregate_rate(args.steps, world, D.max_over_ranks(h0.elapsed_time(h1)))

    # roofline: the inner solve's FP32 K1 (SpMV + p.Ap) on the FP32 copy
    A32 = A.CastTo(np.float32)  # the same FP32 copy the solver makes, tuned the same way
    A32.tune()
    b32 = lmp.B200_lVector.from_numpy(s.b.astype(np.float32), platform=plat, dtype=np.float32)
    x32 = lmp.B200_lVector(n, platform=plat, dtype=np.float32)
    sv32 = lmp.setup_CG_solver(maxits=1000, atol=0.0, rtol=1e-12, dtol=1e8, use_precond=True)
    sv32.SetupOperator(A32)
    sv32._ensure()
    ms3 = (C.c_double * 3)()
    for _ in range(2):  # the first call warms the GPU up after the host-bound e2e loop
        x32.Zeros()
        lib.b200la_cg_profile(sv32._solver, b32.handle, x32.handle, 20, ms3)
    bytes_spmv = spmv_bytes(n, nnz, 4)
    peak, peak_kind = measured_peak_gbs()
    achieved = bytes_spmv / (ms3[0] / 1e3) / 1e9

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        import oracle
        if oracle.ref_available():
            nthreads = os.cpu_count() or 1
            refc = oracle.RefSystem(s.rowptr, s.col, s.val, impl=oracle.IMPL_OPENMP, nthreads=nthreads)
            r, sec = refc.cg(s.b, maxits=20, atol=0.0, rtol=1e-10, dtol=1e8, precond=True)
            cpu = {"value": 1.0 / (sec / max(r.iters, 1) * pcg_iters), "unit": "solves/s", "cores": nthreads,
                   "kind": "reference", "sample": f"20 of {pcg_iters} FP64 Jacobi-PCG iterations (HiFlow3 lmp "
                                                  f"OPENMP SpMV, {nthreads} threads), scaled to a full solve"}
    if rank == 0:
        print(json.dumps({
            "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
            "config": varcoef3d_config(args, s),
            "details": {"precision": f"FP32 Jacobi-PCG inner solve (FP32 matrix and vectors) inside FP64 "
                                     f"refinement; the FP64 residual replaces the inner one every "
                                     f"{inner_rtol:g}x reduction and the search direction is kept",
                        "refinement_passes": outer, "inner_iters": inner, "parallelism": f"replicas x{world}",
                        "true_rel_residual": true_rel,
                        "error_vs_cpu_oracle": {"value": err, "fp64_jacobi_pcg_at_1e-10": err_pcg,
                                                "reference": err_ref},
                        "fp64_jacobi_pcg": {"value": pcg_value, "unit": "solves/s", "iters": pcg_iters,
                                            "reference_iters": varcoef3d_fp64_iters(args.cells)},
                        "mixed_restarted_each_pass": {"value": restart_value, "unit": "solves/s",
                                                      "inner_iters": restart_iters, "passes": restart_passes,
                                                      "inner_rtol": 1e-5},
                        "plain_fp64_cg": {"value": plain_value, "unit": "solves/s", "iters": plain_iters,
                                          "state": plain_state},
                        "speedup_vs_plain_fp64_cg": value / world / plain_value,
                        "speedup_vs_fp64_pcg": value / world / pcg_value},
            "clocks": clk,
            "e2e": {"value": e2e_value, "unit": "solves/s", "h2d_bytes_per_step": n * 8, "d2h_bytes_per_step": n * 8},
            "gpu_launches": args.steps * (3 * inner + 8 * outer + 4),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": profile_traffic(f"varcoef3d_{args.cells}/f32/spmv"), "peak_source": peak_kind,
                         "kernel": "cg_spmv_kernel<float> (inner SpMV fused with p.Ap)",
                         "algorithmic_bytes": bytes_spmv,
                         "kernel_ms": {"spmv_dot": ms3[0], "update": ms3[1], "direction": ms3[2]},
                         **dram_rate(profile_traffic(f"varcoef3d_{args.cells}/f32/spmv"), ms3[0], peak)},
            "cpu_baseline": cpu}))


# ----------------------------------------------------------------- more solvers on the poisson3d matrix
BICG_METRIC = "BiCGSTAB (right Jacobi) solves/s at 1e-10 rel. residual, FP64, 3D Q1 Poisson"
JACOBI_METRIC = "Jacobi smoother sweeps/s (SmoothNormal), FP64, 3D Q1 Poisson"
JACOBI_SWEEPS = 100


def _ref_unavailable():
    import oracle
    if not oracle.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built (reference sources absent)"}))
        return True
    return False


def run_reference_bicgstab(args, rank):
    import oracle
    from ba_b200 import problems as P
    if _ref_unavailable():
        return
    s = P.poisson_3d(args.cells)
    counts = json.load(open(COUNTS)) if os.path.exists(COUNTS) else {}
    full = counts.get(f"poisson3d_{args.cells}/bicgstab_jacobi/rtol1e-10", {}).get("iters", 20)
    nthreads = os.cpu_count() or 1
    sample, per_iter = 10, []
    for step in range(args.warmup + args.steps):
        r, _ = oracle.ref_bicgstab(s.rowptr, s.col, s.val, s.b, maxits=sample, atol=0.0, rtol=1e-10,
                                   dtol=1e8, precond=True, impl=oracle.IMPL_OPENMP, nthreads=nthreads)
        if step >= args.warmup:
            per_iter.append(r.seconds / max(r.iters, 1))
    value = 1.0 / (statistics.median(per_iter) * full)
    print(json.dumps({
        "impl": "reference", "metric": BICG_METRIC, "value": value, "unit": "solves/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 / value, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"fp64 bicgstab + right jacobi, 3d q1 poisson {args.cells}^3 cells, rel 1e-10",
                   "n": s.n, "nnz": s.nnz, "parallelism": f"cpu openmp x{nthreads}"},
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": nthreads, "kind": "reference",
                         "sample": f"{sample} of {full} iterations of one solve per step (HiFlow3 lmp OPENMP "
                                   f"classes, BiCGSTAB<LAD> restated over them), scaled"},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))


def run_reference_jacobi(args, rank):
    import oracle
    from ba_b200 import problems as P
    if _ref_unavailable():
        return
    s = P.poisson_3d(args.cells)
    nthreads = os.cpu_count() or 1
    sample, rates = 5, []
    for step in range(args.warmup + args.steps):
        r = oracle.ref_jacobi(s.rowptr, s.col, s.val, s.b, mode=oracle.JACOBI_SMOOTH_NORMAL, smooth_iter=sample,
                              impl=oracle.IMPL_OPENMP, nthreads=nthreads)
        if step >= args.warmup:
            rates.append(r.iters / r.seconds)
    value = statistics.median(rates)
    print(json.dumps({
        "impl": "reference", "metric": JACOBI_METRIC, "value": value, "unit": "sweeps/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * JACOBI_SWEEPS / value,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"fp64 jacobi smoothing, 3d q1 poisson {args.cells}^3 cells", "n": s.n,
                   "nnz": s.nnz, "parallelism": f"cpu openmp x{nthreads}"},
        "cpu_baseline": {"value": value, "unit": "sweeps/s", "cores": nthreads, "kind": "reference",
                         "sample": f"{sample} sweeps per step (HiFlow3 lmp OPENMP classes, Jacobi<LAD> "
                                   f"DoNormalIteration restated over them)"},
        "e2e": {"value": value, "unit": "sweeps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))


def _c2_setup(args, local_rank, torch):
    from ba_b200 import lmp
    from ba_b200 import problems as P
    plat = lmp.Platform(local_rank)
    stream = work_stream(torch)
    plat.set_stream(stream.cuda_stream)
    s = P.poisson_3d(args.cells)
    A = lmp.B200_CSR_lMatrix(s.rowptr, s.col, s.val, platform=plat)
    fmt, prm, _ = A.tune()
    b = lmp.B200_lVector.from_numpy(s.b, platform=plat)
    x = lmp.B200_lVector(s.n, platform=plat)
    return plat, stream, s, A, fmt, prm, b, x


def _timed(args, stream, torch, barrier, local_rank, step):
    for _ in range(args.warmup):
        step()
    clocks = ClockSampler(local_rank)
    barrier()
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    e1.synchronize()
    barrier()
    return D.max_over_ranks(e0.elapsed_time(e1)), clocks.stop()


def _timed_e2e(args, stream, torch, barrier, b, x, n, step):
    import ctypes as C
    from ba_b200._lib import load
    lib = load()
    bh = torch.from_numpy(np.zeros(n)).pin_memory()
    bh.copy_(torch.from_numpy(b.numpy()))
    xh = torch.empty(n, dtype=torch.float64).pin_memory()
    barrier()
    h0, h1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    h0.record(stream)
    for _ in range(args.steps):
        lib.b200la_vec_upload(b.handle, C.c_void_p(bh.data_ptr()), n)
        step()
        lib.b200la_vec_download(x.handle, C.c_void_p(xh.data_ptr()), n)
    h1.record(stream)
    h1.synchronize()
    return D.max_over_ranks(h0.elapsed_time(h1))


def run_bicgstab(args, rank, local_rank, world, torch, dist, barrier):
    from ba_b200 import lmp
    from ba_b200._lib import FORMAT_NAMES
    plat, stream, s, A, fmt, prm, b, x = _c2_setup(args, local_rank, torch)
    n, nnz = s.n, s.nnz
    solver = lmp.BiCGSTAB()
    solver.InitControl(20000, 0.0, 1e-10, 1e8)
    solver.SetupOperator(A)
    pc = lmp.PreconditionerBlockJacobiStand()
    pc.Init_Jacobi()
    solver.SetupPreconditioner(pc)

    def step():
        x.Zeros()
        assert solver.Solve(b, x) == lmp.kSolverSuccess
    ms_max, clk = _timed(args, stream, torch, barrier, local_rank, step)
    iters = solver.iter()
    value = D.aggregate_rate(args.steps, world, ms_max)
    e2e_value = D.aggregate_rate(args.steps, world, _timed_e2e(args, stream, torch, barrier, b, x, n, step))
    for _ in range(2):  # the first call warms the GPU up after the host-bound e2e loop
        x.Zeros()
        ms = solver.profile(b, x, 20)
    bytes_b1 = spmv_bytes(n, nnz, 8) + n * 8
    peak, peak_kind = measured_peak_gbs()
    achieved = bytes_b1 / (ms[0] / 1e3) / 1e9
    key = f"poisson3d_{args.cells}/f64/bicgstab_spmv_q"
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        import oracle
        if oracle.ref_available():
            nthreads = os.cpu_count() or 1
            r, _ = oracle.ref_bicgstab(s.rowptr, s.col, s.val, s.b, maxits=10, atol=0.0, rtol=1e-10, dtol=1e8,
                                       precond=True, impl=oracle.IMPL_OPENMP, nthreads=nthreads)
            cpu = {"value": 1.0 / (r.seconds / max(r.iters, 1) * iters), "unit": "solves/s", "cores": nthreads,
                   "kind": "reference", "sample": f"10 of {iters} iterations of one solve (HiFlow3 lmp OPENMP "
                                                  f"classes, {nthreads} threads), scaled to a full solve"}
    if rank == 0:
        print(json.dumps({
            "metric": BICG_METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"fp64 bicgstab + right jacobi, 3d q1 poisson {args.cells}^3 cells, rel 1e-10",
                       "n": n, "nnz": nnz, "iters_per_solve": iters, "restarts": solver.restarts(),
                       "parallelism": f"replicas x{world}", "spmv_schedule": FORMAT_NAMES[fmt] + f"/{prm}",
                       "l2": "inputs larger than L2 (matrix 685 MB streamed twice per iteration)"},
            "clocks": clk,
            "e2e": {"value": e2e_value, "unit": "solves/s", "h2d_bytes_per_step": n * 8, "d2h_bytes_per_step": n * 8},
            "gpu_launches": args.steps * 5 * (iters + 1),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": profile_traffic(key), "peak_source": peak_kind,
                         "kernel": "bicg_spmv_q_kernel (A q fused with Ap.r0, Ap.Ap)", "algorithmic_bytes": bytes_b1,
                         "kernel_ms": dict(zip(("spmv_q", "s_update", "spmv_s", "xr_update", "direction"), ms)),
                         **dram_rate(profile_traffic(key), ms[0], peak)},
            "cpu_baseline": cpu}))


def run_jacobi(args, rank, local_rank, world, torch, dist, barrier):
    from ba_b200 import lmp
    from ba_b200._lib import FORMAT_NAMES
    plat, stream, s, A, fmt, prm, b, x = _c2_setup(args, local_rank, torch)
    n, nnz = s.n, s.nnz
    j = lmp.Jacobi()
    j.SetupOperator(A)
    j.SetSolveMode(2)
    j.SetNumIter(JACOBI_SWEEPS)

    def step():
        x.Zeros()
        assert j.Solve(b, x) == lmp.kSolverSuccess
    ms_max, clk = _timed(args, stream, torch, barrier, local_rank, step)
    value = D.aggregate_rate(args.steps * JACOBI_SWEEPS, world, ms_max)
    e2e_value = D.aggregate_rate(args.steps * JACOBI_SWEEPS, world,
                                 _timed_e2e(args, stream, torch, barrier, b, x, n, step))
    for _ in range(2):  # the first call warms the GPU up after the host-bound e2e loop
        x.Zeros()
        ms = j.profile(b, x, 20)
    bytes_sweep = spmv_bytes(n, nnz, 8) + 2 * n * 8
    peak, peak_kind = measured_peak_gbs()
    achieved = bytes_sweep / (ms[0] / 1e3) / 1e9
    key = f"poisson3d_{args.cells}/f64/jacobi_sweep"
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        import oracle
        if oracle.ref_available():
            nthreads = os.cpu_count() or 1
            r = oracle.ref_jacobi(s.rowptr, s.col, s.val, s.b, mode=oracle.JACOBI_SMOOTH_NORMAL, smooth_iter=5,
                                  impl=oracle.IMPL_OPENMP, nthreads=nthreads)
            cpu = {"value": r.iters / r.seconds, "unit": "sweeps/s", "cores": nthreads, "kind": "reference",
                   "sample": f"5 sweeps (HiFlow3 lmp OPENMP classes, {nthreads} threads)"}
    if rank == 0:
        print(json.dumps({
            "metric": JACOBI_METRIC, "value": value, "unit": "sweeps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"fp64 jacobi smoothing ({JACOBI_SWEEPS} sweeps per step), 3d q1 poisson "
                                   f"{args.cells}^3 cells", "n": n, "nnz": nnz, "parallelism": f"replicas x{world}",
                       "spmv_schedule": FORMAT_NAMES[fmt] + f"/{prm}",
                       "l2": "inputs larger than L2 (matrix 685 MB streamed per sweep)"},
            "clocks": clk,
            "e2e": {"value": e2e_value, "unit": "sweeps/s", "h2d_bytes_per_step": n * 8, "d2h_bytes_per_step": n * 8},
            "gpu_launches": args.steps * JACOBI_SWEEPS,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": profile_traffic(key), "peak_source": peak_kind,
                         "kernel": "jacobi_sweep_kernel (r = b - A x_k, ||r||, x_k+1 = x_k + inv_D r)",
                         "algorithmic_bytes": bytes_sweep, "kernel_ms": ms[0],
                         **dram_rate(profile_traffic(key), ms[0], peak)},
            "cpu_baseline": cpu}))


GMRES_METRIC = "GMRES(100) (right Jacobi) solves/s at 1e-10 rel. residual, FP64, 3D Q1 Poisson"
GMRES_BASIS = 100


def run_reference_gmres(args, rank):
    import oracle
    from ba_b200 import problems as P
    if _ref_unavailable():
        return
    s = P.poisson_3d(args.cells)
    counts = json.load(open(COUNTS)) if os.path.exists(COUNTS) else {}
    full = counts.get(f"poisson3d_{args.cells}/gmres{GMRES_BASIS}_jacobi/rtol1e-10", {}).get("iters", GMRES_BASIS)
    nthreads = os.cpu_count() or 1
    per_iter = []
    # one whole cycle per step: the Gram-Schmidt cost grows within a cycle
    for step in range(max(1, args.warmup // 3) + args.steps):
        r = oracle.ref_gmres(s.rowptr, s.col, s.val, s.b, size_basis=GMRES_BASIS, maxits=GMRES_BASIS, atol=0.0,
                             rtol=1e-10, dtol=1e8, precond=True, impl=oracle.IMPL_OPENMP, nthreads=nthreads)
        if step >= max(1, args.warmup // 3):
            per_iter.append(r.seconds / max(r.iters, 1))
    value = 1.0 / (statistics.median(per_iter) * full)
    print(json.dumps({
        "impl": "reference", "metric": GMRES_METRIC, "value": value, "unit": "solves/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 / value, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"fp64 gmres({GMRES_BASIS}) + right jacobi, 3d q1 poisson {args.cells}^3 cells, "
                               f"rel 1e-10", "n": s.n, "nnz": s.nnz, "parallelism": f"cpu openmp x{nthreads}"},
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": nthreads, "kind": "reference",
                         "sample": f"the first {GMRES_BASIS}-step cycle of one solve per step (HiFlow3 lmp OPENMP "
                                   f"classes, GMRES<LAD> restated over them), scaled to {full} steps"},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))


def run_gmres(args, rank, local_rank, world, torch, dist, barrier):
    from ba_b200 import lmp
    from ba_b200._lib import FORMAT_NAMES
    plat, stream, s, A, fmt, prm, b, x = _c2_setup(args, local_rank, torch)
    n, nnz = s.n, s.nnz
    solver = lmp.GMRES()
    solver.InitParameter(GMRES_BASIS, "RightPreconditioning")
    solver.InitControl(20000, 0.0, 1e-10, 1e8)
    solver.SetupOperator(A)
    pc = lmp.PreconditionerBlockJacobiStand()
    pc.Init_Jacobi()
    solver.SetupPreconditioner(pc)

    def step():
        x.Zeros()
        assert solver.Solve(b, x) == lmp.kSolverSuccess
    ms_max, clk = _timed(args, stream, torch, barrier, local_rank, step)
    iters = solver.iter()
    value = D.aggregate_rate(args.steps, world, ms_max)
    e2e_value = D.aggregate_rate(args.steps, world, _timed_e2e(args, stream, torch, barrier, b, x, n, step))
    # kernel times over the first cycle (the Arnoldi step grows with j)
    x.Zeros()
    ms = solver.profile(b, x, GMRES_BASIS)
    bytes_spmv = spmv_bytes(n, nnz, 8) + n * 8
    avg_j = (GMRES_BASIS - 1) / 2.0
    # w stays in shared memory for the step: V_0..V_j read once each, w and
    # invD read, V_{j+1} and z written
    bytes_arnoldi = int((avg_j + 1 + 4) * n * 8)
    peak, peak_kind = measured_peak_gbs()
    achieved = bytes_spmv / (ms[2] / 1e3) / 1e9
    key = f"poisson3d_{args.cells}/f64/gmres_spmv"
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        import oracle
        if oracle.ref_available():
            nthreads = os.cpu_count() or 1
            r = oracle.ref_gmres(s.rowptr, s.col, s.val, s.b, size_basis=GMRES_BASIS, maxits=GMRES_BASIS, atol=0.0,
                                 rtol=1e-10, dtol=1e8, precond=True, impl=oracle.IMPL_OPENMP, nthreads=nthreads)
            cpu = {"value": 1.0 / (r.seconds / max(r.iters, 1) * iters), "unit": "solves/s", "cores": nthreads,
                   "kind": "reference", "sample": f"the first {GMRES_BASIS}-step cycle (HiFlow3 lmp OPENMP classes, "
                                                  f"{nthreads} threads), scaled to {iters} steps"}
    if rank == 0:
        print(json.dumps({
            "metric": GMRES_METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"fp64 gmres({GMRES_BASIS}) + right jacobi, 3d q1 poisson {args.cells}^3 cells, "
                                   f"rel 1e-10", "n": n, "nnz": nnz, "iters_per_solve": iters,
                       "parallelism": f"replicas x{world}", "spmv_schedule": FORMAT_NAMES[fmt] + f"/{prm}",
                       "l2": "inputs larger than L2 (matrix 685 MB streamed per step, basis 1.7 GB)"},
            "clocks": clk,
            "e2e": {"value": e2e_value, "unit": "solves/s", "h2d_bytes_per_step": n * 8, "d2h_bytes_per_step": n * 8},
            "gpu_launches": args.steps * (4 * iters + 5),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": profile_traffic(key), "peak_source": peak_kind,
                         "kernel": "gm_spmv_kernel (w = A P v_j fused with w.V0)", "algorithmic_bytes": bytes_spmv,
                         "kernel_ms": dict(zip(("cycle_update", "restart", "spmv", "arnoldi"), ms)),
                         "arnoldi": {"algorithmic_bytes_mean": bytes_arnoldi,
                                     "gbs": bytes_arnoldi / (ms[3] / 1e3) / 1e9,
                                     "frac": bytes_arnoldi / (ms[3] / 1e3) / 1e9 / peak,
                                     "note": "mean over the first cycle, w resident in shared memory: V_0..V_j "
                                             "read once each, w and invD read, V_{j+1} and z written; the step "
                                             "waits on j+1 grid barriers"},
                         **dram_rate(profile_traffic(key), ms[2], peak)},
            "cpu_baseline": cpu}))


COO_METRIC = "TransformFromCOO conversions/s (device COO -> CSR), 3D Q1 Poisson triplets in random order"


def _coo_triplets(cells):
    from ba_b200 import problems as P
    s = P.poisson_3d(cells)
    rows = np.repeat(np.arange(s.n, dtype=np.int32), np.diff(s.rowptr))
    perm = np.random.default_rng(20240603).permutation(s.nnz)
    return s, rows[perm], s.col[perm], s.val[perm]


def run_reference_coo(args, rank):
    import oracle
    if _ref_unavailable():
        return
    s, r, c, v = _coo_triplets(args.cells)
    secs = []
    for step in range(1 + args.steps):
        t = time.perf_counter()
        oracle.ref_coo_to_csr(s.n, s.n, r, c, v)
        if step >= 1:
            secs.append(time.perf_counter() - t)
    value = 1.0 / statistics.median(secs)
    print(json.dumps({
        "impl": "reference", "metric": COO_METRIC, "value": value, "unit": "conversions/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": 1, "ms_per_step": 1e3 / value, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"TransformFromCOO of the 3d q1 poisson {args.cells}^3 matrix, triplets shuffled",
                   "n": s.n, "nnz": s.nnz, "parallelism": "cpu, 1 thread (the reference's coo_2_csr is serial)"},
        "cpu_baseline": {"value": value, "unit": "conversions/s", "cores": 1, "kind": "reference",
                         "sample": "whole conversions, host arrays in, CSR out (copied from the matrix)"},
        "e2e": {"value": value, "unit": "conversions/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))


def run_coo(args, rank, local_rank, world, torch, dist, barrier):
    from ba_b200 import lmp
    plat = lmp.Platform(local_rank)
    stream = work_stream(torch)
    plat.set_stream(stream.cuda_stream)
    s, r, c, v = _coo_triplets(args.cells)
    dev = [torch.from_numpy(a).cuda() for a in (r, c, v)]
    torch.cuda.synchronize()

    def step():
        A = lmp.B200_CSR_lMatrix.TransformFromCOO(*dev, s.n, s.n, platform=plat)
        A.Clear()
    ms_max, clk = _timed(args, stream, torch, barrier, local_rank, step)
    value = D.aggregate_rate(args.steps, world, ms_max)
    # e2e: triplets from pinned host memory in, CSR back into pinned host memory
    def pinned(a):
        t = torch.empty(a.shape, dtype=getattr(torch, a.dtype.name), pin_memory=True)
        t.numpy()[...] = a
        return t
    hin = [pinned(a) for a in (r, c, v)]
    hout = [torch.empty(n, dtype=dt, pin_memory=True)
            for n, dt in ((s.n + 1, torch.int32), (s.nnz, torch.int32), (s.nnz, torch.float64))]
    hin_np, hout_np = [t.numpy() for t in hin], tuple(t.numpy() for t in hout)
    barrier()
    h0, h1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    h0.record(stream)
    for _ in range(args.steps):
        A = lmp.B200_CSR_lMatrix.TransformFromCOO(*hin_np, s.n, s.n, platform=plat)
        A.csr(out=hout_np)
        A.Clear()
    h1.record(stream)
    h1.synchronize()
    e2e_value = D.aggregate_rate(args.steps, world, D.max_over_ranks(h0.elapsed_time(h1)))
    ok = all(np.array_equal(a, b) for a, b in zip(hout_np, (s.rowptr, s.col, s.val)))
    A = lmp.B200_CSR_lMatrix.TransformFromCOO(*dev, s.n, s.n, platform=plat)
    ok = ok and all(np.array_equal(a, b) for a, b in zip(A.csr(), (s.rowptr, s.col, s.val)))
    A.Clear()
    # algorithmic bytes: read the triplets (16 B), write col + val (12 B) and the row pointer
    alg = s.nnz * (4 + 4 + 8) + s.nnz * (4 + 8) + (s.n + 1) * 4
    peak, peak_kind = measured_peak_gbs()
    achieved = alg / (ms_max / args.steps / 1e3) / 1e9
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        import oracle
        if oracle.ref_available():
            t = time.perf_counter()
            oracle.ref_coo_to_csr(s.n, s.n, r, c, v)
            cpu = {"value": 1.0 / (time.perf_counter() - t), "unit": "conversions/s", "cores": 1,
                   "kind": "reference", "sample": "one whole conversion (the reference's coo_2_csr is serial)"}
    if rank == 0:
        print(json.dumps({
            "metric": COO_METRIC, "value": value, "unit": "conversions/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"TransformFromCOO of the 3d q1 poisson {args.cells}^3 matrix, triplets shuffled",
                       "n": s.n, "nnz": s.nnz, "matches_generator_csr": ok, "parallelism": f"replicas x{world}",
                       "l2": "inputs larger than L2 (913 MB of triplets)",
                       "launches": "6 of ours per conversion (check, iota, row offsets, gather, row sort, long "
                                   "rows) and 5 of the CUB radix sort",
                       "e2e_host_buffers": "pinned"},
            "clocks": clk,
            "e2e": {"value": e2e_value, "unit": "conversions/s", "h2d_bytes_per_step": s.nnz * 16,
                    "d2h_bytes_per_step": s.nnz * 12 + (s.n + 1) * 4},
            "gpu_launches": args.steps * 6,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": None, "peak_source": peak_kind,
                         "kernel": "whole conversion (check, radix sort by row, row offsets, gather, row sort)",
                         "algorithmic_bytes": alg,
                         "note": "the radix sort moves the keys and positions several times; the algorithmic "
                                 "bytes count one read of the triplets and one write of the CSR"},
            "cpu_baseline": cpu}))


def main():
    args = parse()
    rank, local_rank, world = dist_env()
    if args.impl == "reference":
        if rank == 0:
            {"batch": run_reference_batch, "poisson3d": run_reference_poisson3d,
             "varcoef3d": run_reference_varcoef3d, "serve": run_reference_serve,
             "bicgstab": run_reference_bicgstab, "jacobi": run_reference_jacobi,
             "gmres": run_reference_gmres, "coo": run_reference_coo}[args.workload](args, rank)
        return
    import datetime

    import torch
    import torch.distributed as dist

    from ba_b200 import load
    torch.cuda.set_device(local_rank)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    load()
    fn = {"batch": run_batch, "poisson3d": run_poisson3d, "varcoef3d": run_varcoef3d,
          "serve": run_serve, "bicgstab": run_bicgstab, "jacobi": run_jacobi, "gmres": run_gmres,
          "coo": run_coo}[args.workload]
    fn(args, rank, local_rank, world, torch, dist, barrier)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
