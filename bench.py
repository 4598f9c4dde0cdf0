#!/usr/bin/env python
"""Benchmark of the Jacobi-PCG hot path on B200 (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload poisson3d]

Workload "poisson3d": FP64 Jacobi-PCG on 3D Q1 Poisson, 128^3 hex cells
(2,146,689 DOFs, 57,066,625 nnz, FP64 values, int32 indices), Dirichlet
boundary, seeded U[0,1) RHS, rel. residual 1e-10.  A step is one full solve;
the metric is solves/s.  The matrix (685 MB) is larger than L2, so each
iteration streams it from HBM.

Multi-GPU: every rank solves its own copy of the system (replicas; the path
has no exchange step for independent solves), value = all ranks' solves / the
slowest rank's time.

--impl reference times the reference's own CPU implementation (HiFlow3 lmp
sources compiled into oracle/_ref: OPENMP CSR SpMV on all host cores, lmp
BLAS-1, lPreconditioner_Jacobi, CG<LAD> recurrence) on the same system, a
bounded sample of iterations per step scaled by the reference's own
iteration count for the full solve (tests/golden/workload_counts.json).
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

METRIC = "PCG solves/s & p50/p99 latency at 1e-8 rel. residual vs plain FP64 GPU CG"
COUNTS = os.path.join(ROOT, "tests", "golden", "workload_counts.json")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="poisson3d", choices=["poisson3d"])
    ap.add_argument("--cells", type=int, default=128)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


def dist_env():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0")),
            int(os.environ.get("WORLD_SIZE", "1")))


def measured_peak_gbs():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        return float(json.load(open(p))["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


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


def run_reference(args, rank: int):
    """The reference CPU implementation, rank 0 only."""
    if rank != 0:
        return
    import oracle
    from ba_b200 import problems as P
    if not oracle.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built (reference sources absent)"}))
        return
    s = P.poisson_3d(args.cells)
    counts = json.load(open(COUNTS)) if os.path.exists(COUNTS) else {}
    key = f"poisson3d_{args.cells}/jacobi/rtol1e-10"
    full_iters = counts.get(key, {}).get("iters")
    nthreads = os.cpu_count() or 1
    ref = oracle.RefSystem(s.rowptr, s.col, s.val, impl=oracle.IMPL_OPENMP, nthreads=nthreads)
    sample_iters = 20
    per_iter = []
    for step in range(args.warmup + args.steps):
        r, sec = ref.cg(s.b, maxits=sample_iters, atol=0.0, rtol=1e-10, dtol=1e8, precond=True)
        if step >= args.warmup:
            per_iter.append(sec / max(r.iters, 1))
    t_iter = statistics.median(per_iter)
    iters = full_iters or sample_iters
    value = 1.0 / (t_iter * iters)
    out = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 / value, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"fp64 jacobi-pcg 3d q1 poisson {args.cells}^3 cells, rel 1e-10",
                   "n": s.n, "nnz": s.nnz, "parallelism": "cpu openmp"},
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": nthreads, "kind": "reference",
                         "sample": f"{sample_iters} of {iters} iterations of one solve per step "
                                   f"(HiFlow3 lmp OPENMP SpMV, {nthreads} threads), scaled to a full solve"},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out))


def cpu_baseline_leg(s, full_iters):
    """Reference CPU CG on the same system (bounded sample, all host threads)."""
    import oracle
    if not oracle.ref_available():
        return None
    nthreads = os.cpu_count() or 1
    ref = oracle.RefSystem(s.rowptr, s.col, s.val, impl=oracle.IMPL_OPENMP, nthreads=nthreads)
    sample_iters = 20
    ref.cg(s.b, maxits=2, atol=0.0, rtol=1e-10, dtol=1e8)
    r, sec = ref.cg(s.b, maxits=sample_iters, atol=0.0, rtol=1e-10, dtol=1e8, precond=True)
    t_iter = sec / max(r.iters, 1)
    ref.close()
    return {"value": 1.0 / (t_iter * full_iters), "unit": "solves/s", "cores": nthreads, "kind": "reference",
            "sample": f"{sample_iters} of {full_iters} iterations of one solve (HiFlow3 lmp OPENMP SpMV, "
                      f"{nthreads} threads), scaled to a full solve"}


def main():
    args = parse()
    rank, local_rank, world = dist_env()
    if args.impl == "reference":
        run_reference(args, rank)
        return

    import torch
    import torch.distributed as dist

    from ba_b200 import lmp
    from ba_b200 import problems as P
    from ba_b200._lib import FMT_SELL, load

    torch.cuda.set_device(local_rank)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    load()
    plat = lmp.Platform(local_rank)
    stream = torch.cuda.current_stream()
    plat.set_stream(stream.cuda_stream)

    s = P.poisson_3d(args.cells)
    n, nnz = s.n, s.nnz
    A = lmp.B200_CSR_lMatrix(s.rowptr, s.col, s.val, platform=plat)
    fmt, prm, tune_us = A.tune()
    b = lmp.B200_lVector.from_numpy(s.b, platform=plat)
    x = lmp.B200_lVector(n, platform=plat)
    rtol = 1e-10
    solver = lmp.setup_CG_solver(maxits=20000, atol=0.0, rtol=rtol, dtol=1e8, use_precond=True)
    solver.SetupOperator(A)
    plain = lmp.setup_CG_solver(maxits=20000, atol=0.0, rtol=rtol, dtol=1e8, use_precond=False)
    plain.SetupOperator(A)

    def step(sv):
        x.Zeros()
        st = sv.Solve(b, x)
        assert st == lmp.kSolverSuccess, st
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
    ms = e0.elapsed_time(e1)
    t = torch.tensor([ms], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    value = world * args.steps / (ms_max / 1e3)

    # plain FP64 GPU CG (SolveNoPrecond recurrence) on the same system: the comparator
    step(plain)
    barrier()
    c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    k_plain = max(2, args.steps // 2)
    c0.record(stream)
    for _ in range(k_plain):
        step(plain)
    c1.record(stream)
    c1.synchronize()
    plain_value = k_plain / (c0.elapsed_time(c1) / 1e3)
    plain_iters = plain.iter()

    # end to end through the public API: H2D of the RHS from pinned memory,
    # solve, D2H of the solution, every step.
    bh = torch.from_numpy(s.b).pin_memory()
    xh = torch.empty(n, dtype=torch.float64).pin_memory()
    import ctypes as C
    lib = load()
    barrier()
    h0, h1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    h0.record(stream)
    for _ in range(args.steps):
        lib.b200la_vec_upload(b.handle, C.c_void_p(bh.data_ptr()), n)
        step(solver)
        lib.b200la_vec_download(x.handle, C.c_void_p(xh.data_ptr()), n)
    h1.record(stream)
    h1.synchronize()
    te = torch.tensor([h0.elapsed_time(h1)], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    e2e_value = world * args.steps / (float(te.item()) / 1e3)

    # roofline of the dominant kernel (SpMV + p.Ap), timed live with CUDA events
    ms3 = (C.c_double * 3)()
    x.Zeros()
    lib.b200la_cg_profile(solver._solver, b.handle, x.handle, 20, ms3)
    t_spmv = ms3[0] / 1e3
    bytes_spmv = spmv_bytes(n, nnz, 8)
    peak, peak_kind = measured_peak_gbs()
    achieved = bytes_spmv / t_spmv / 1e9
    traffic = None
    prof = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(prof):
        traffic = json.load(open(prof)).get(f"poisson3d_{args.cells}/f64/spmv")

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        counts = json.load(open(COUNTS)) if os.path.exists(COUNTS) else {}
        full = counts.get(f"poisson3d_{args.cells}/jacobi/rtol1e-10", {}).get("iters", iters)
        cpu = cpu_baseline_leg(s, full)

    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"fp64 jacobi-pcg 3d q1 poisson {args.cells}^3 cells, rel 1e-10",
                       "n": n, "nnz": nnz, "iters_per_solve": iters, "parallelism": f"replicas x{world}",
                       "spmv_schedule": ("sell" if fmt == FMT_SELL else "csr") + f"/{prm}",
                       "l2": "inputs larger than L2 (matrix 685 MB streamed per iteration)",
                       "plain_fp64_cg": {"value": plain_value, "unit": "solves/s", "iters_per_solve": plain_iters}},
            "clocks": clk,
            "e2e": {"value": e2e_value, "unit": "solves/s", "h2d_bytes_per_step": n * 8, "d2h_bytes_per_step": n * 8},
            "gpu_launches": args.steps * (1 + 3 * iters),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": traffic, "peak_source": peak_kind,
                         "kernel": "cg_spmv_kernel (SpMV fused with p.Ap)", "algorithmic_bytes": bytes_spmv,
                         "kernel_ms": {"spmv_dot": ms3[0], "update": ms3[1], "direction": ms3[2]}},
            "cpu_baseline": cpu,
        }
        print(json.dumps(out))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
