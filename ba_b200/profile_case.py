"""Profiling driver: runs the path's kernels on one standard system as plain
launches (no CUDA graph), so a profiler sees every launch on its own.

    python -m ba_b200.profile_case [--cells 128] [--dim 3] [--dtype f64|f32]
                                   [--spmv-reps 3] [--cg-iters 3] [--schedule tune|csr/8|sell/1]
    python -m ba_b200.profile_case --sell-table [--dtype f64|f32]

With --solver jacobi|bicgstab|gmres: after the SpMV launches, runs
`--cg-iters` passes of that solver's kernels as plain launches
(b200la_solver_profile: one jacobi_sweep_kernel per pass; bicg_spmv_q,
bicg_s, bicg_spmv_s, bicg_update, bicg_direction per pass, the first pass a
restart; gm_update, gm_restart, gm_spmv, gm_arnoldi per pass, the first
pass's gm_restart building V0) instead of the CG kernels.

With --batch N: builds the standard batch of N 2D systems (bench.py's batch
settings; --batch-dim 3: N device-assembled 3D systems instead) and solves it --solves times (default 2; the launches of interest
are those of the last solve; set B200LA_GRAPHS=0 so the kernels launch one by
one), compacting every --chunk passes, with --adaptive item shrinking.  With --profile-only the
solves are skipped: one restart pass (K1 K2 K3) is followed by three timed
inner passes (K1 K2 K3 each), the launches a profiler should capture.

Launch order: the tuner's SpMV launches (unless a schedule is given), then
`--spmv-reps` plain SpMV launches (spmv_kernel), then the CG init kernel and
`--cg-iters` iterations of cg_spmv_kernel, cg_update_kernel and
cg_direction_kernel.  Prints the CUDA-event time of each kernel.
"""
from __future__ import annotations

import argparse
import ctypes as C
import time

import numpy as np

from . import lmp
from . import problems as P
from ._lib import FMT_CSR, FMT_SELL, FMT_SELL16, FMT_STENCIL, FORMAT_NAMES, call, load


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--cells", type=int, default=128)
    ap.add_argument("--dim", type=int, default=3)
    ap.add_argument("--dtype", default="f64", choices=["f64", "f32"])
    ap.add_argument("--spmv-reps", type=int, default=3)
    ap.add_argument("--cg-iters", type=int, default=3)
    ap.add_argument("--schedule", default="tune")
    ap.add_argument("--sigma", type=float, default=0.0)
    ap.add_argument("--solver", default="cg", choices=["cg", "jacobi", "bicgstab", "gmres"])
    ap.add_argument("--basis", type=int, default=100, help="gmres: Krylov basis size")
    ap.add_argument("--batch", type=int, default=0,
                    help="instead: solve a batch of this many 2D systems (n~logU[16,256], sigma 1) twice")
    ap.add_argument("--chunk", type=int, default=64, help="batch: passes per graph launch (compaction in between)")
    ap.add_argument("--batch-dim", type=int, default=2, choices=[2, 3],
                    help="batch: 2 = bench.py's 2D batch; 3 = 3D Q1 systems of 40..90 cells per axis (cycled), "
                         "assembled on the device")
    ap.add_argument("--adaptive", action="store_true",
                    help="batch: shrink items while the running systems give a kernel's warps fewer than one each")
    ap.add_argument("--solves", type=int, default=2, help="batch: solves of the whole batch (timed one by one)")
    ap.add_argument("--tile-rows", type=int, default=0)
    ap.add_argument("--index-bits", type=int, default=0, choices=[0, 16, 32],
                    help="batch: sliced-ELL columns (0 = values only when every row fits the system's stencil, "
                         "else int16 offsets when they fit; 16 = int16 offsets when they fit; 32 = int32)")
    ap.add_argument("--items", default="", help="batch: K1,K2,K3 item rows instead of tuning")
    ap.add_argument("--profile-only", action="store_true",
                    help="batch: skip the solves; time one inner pass kernel by kernel (b200la_batch_profile_pass)")
    ap.add_argument("--sell-table", action="store_true",
                    help="instead: time every SpMV schedule (CSR lane groups, SELL-C-sigma with C 8/16/32, sigma "
                         "1/1024, widths 1/2/4, int32/int16 columns; the values-only stencil copy with widths 1/2/4) on "
                         "three matrices and print a table")
    a = ap.parse_args()
    if a.sell_table:
        return sell_table(a)
    if a.batch:
        return batch_case(a)
    dt = np.float64 if a.dtype == "f64" else np.float32
    s = P.q1_system(a.dim, a.cells, 20240602, a.sigma)
    plat = lmp.init_platform(0)
    A = lmp.B200_CSR_lMatrix(s.rowptr, s.col, s.val, platform=plat, dtype=dt)
    if a.schedule == "tune":
        fmt, prm, us = A.tune()
    else:
        kind, prm = a.schedule.split("/")
        fmt, prm = {"sell": FMT_SELL, "sell16": FMT_SELL16, "csr": FMT_CSR, "stencil": FMT_STENCIL}[kind], int(prm)
        A.set_format(fmt, prm)
        us = float("nan")
    x = lmp.B200_lVector.from_numpy(s.b.astype(dt), platform=plat, dtype=dt)
    y = x.CloneWithoutContent()
    plat.synchronize()
    t = time.perf_counter()
    for _ in range(a.spmv_reps):
        A.VectorMult(x, y)
    plat.synchronize()
    spmv_ms = (time.perf_counter() - t) * 1e3 / max(a.spmv_reps, 1)
    sv = 8 if dt == np.float64 else 4
    alg = s.nnz * (sv + 4) + (s.n + 1) * 4 + 2 * s.n * sv
    if a.solver != "cg":
        return solver_case(a, s, A, dt, fmt, prm, us, alg, sv)
    solver = lmp.setup_CG_solver(maxits=100000, atol=0.0, rtol=1e-12, dtol=1e8)
    solver.SetupOperator(A)
    solver._ensure()
    b = lmp.B200_lVector.from_numpy(s.b.astype(dt), platform=plat, dtype=dt)
    x0 = lmp.B200_lVector(s.n, platform=plat, dtype=dt)
    ms = (C.c_double * 3)()
    call("b200la_cg_profile", solver._solver, b.handle, x0.handle, a.cg_iters, ms)
    print(f"system n={s.n} nnz={s.nnz} dtype={a.dtype} schedule={FORMAT_NAMES[fmt]}/{prm} "
          f"tuned_us={us:.1f}")
    print(f"spmv wall {spmv_ms:.3f} ms/launch; cg kernels ms: spmv_dot {ms[0]:.4f} update {ms[1]:.4f} "
          f"direction {ms[2]:.4f}; spmv algorithmic bytes {alg} -> {alg / ms[0] / 1e6:.1f} GB/s")
    load()


def ragged_system(n: int, seed: int = 11):
    """A banded matrix with power-law row lengths (1..200 entries, mean ~7,
    a few long rows among many short ones, columns within 5,000 of the row):
    the case SELL-C-sigma's sorting is for."""
    u = P.uniform01(seed, n, stream=1)
    deg = np.minimum(1 + (3.0 * ((1.0 - u) ** (-1.0 / 1.5) - 1.0)).astype(np.int64), 200)
    rowptr = np.zeros(n + 1, np.int64)
    np.cumsum(deg, out=rowptr[1:])
    nnz = int(rowptr[-1])
    rows = np.repeat(np.arange(n, dtype=np.int64), deg)
    off = (P.uniform01(seed, nnz, stream=2) * 10001).astype(np.int64) - 5000
    cols = np.clip(rows + off, 0, n - 1)
    order = np.lexsort((cols, rows))
    cols = cols[order]
    val = P.uniform01(seed, nnz, stream=3) - 0.5
    return P.CSRSystem(0, 0, rowptr.astype(np.int32), cols.astype(np.int32), val, P.uniform01(seed, n, stream=4),
                       np.zeros(n, bool), f"ragged_{n}")


def sell_table(a):
    """Every SpMV schedule on three matrices, CUDA-event timed (20 launches
    after 3 warm-ups), as a markdown table: microseconds per SpMV, padding of
    the sliced copy, algorithmic GB/s; then the tuner's pick."""
    import torch
    dt = np.float64 if a.dtype == "f64" else np.float32
    sv = 8 if dt == np.float64 else 4
    plat = lmp.init_platform(0)
    st = torch.cuda.Stream()  # not the legacy default stream: handle 0 selects the context's own stream
    torch.cuda.set_stream(st)
    plat.set_stream(st.cuda_stream)
    cases = [P.q1_system(2, 1024, 20240601, 1.0, "q1_2d_1024_s1"), P.q1_system(3, 128, 20240602, 2.0, "q1_3d_128_s2"),
             ragged_system(2_000_000)]
    print(f"| matrix | schedule | C | sigma | us | padding | GB/s |")
    print(f"|---|---|---:|---:|---:|---:|---:|")
    for s in cases:
        A = lmp.B200_CSR_lMatrix(s.rowptr, s.col, s.val, platform=plat, dtype=dt)
        x = lmp.B200_lVector.from_numpy(s.b.astype(dt), platform=plat, dtype=dt)
        y = x.CloneWithoutContent()
        alg = s.nnz * (sv + 4) + (s.n + 1) * 4 + 2 * s.n * sv
        rows = []

        def timed():
            for _ in range(3):
                A.VectorMult(x, y)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            for _ in range(20):
                A.VectorMult(x, y)
            e1.record(st)
            e1.synchronize()
            return e0.elapsed_time(e1) * 1e3 / 20
        for g in (2, 4, 8, 16, 32):
            A.set_format(FMT_CSR, g)
            rows.append((f"csr/{g}", "", "", timed(), ""))
        for col16 in (False, True):
            for sigma in (1, 1024):
                for c in (32, 16, 8):
                    for w in (1, 2, 4):
                        try:
                            A.set_sell(c, sigma, w, col16)
                        except lmp.B200LAError:
                            continue
                        padded = A.sell_padded()
                        rows.append((f"{'sell16' if col16 else 'sell'}/{w}", c, sigma, timed(),
                                     f"{padded / s.nnz - 1:.1%}"))
        for w in (1, 2, 4):
            try:
                A.set_format(FMT_STENCIL, w)
            except lmp.B200LAError:
                continue
            rows.append((f"stencil/{w}", 32, 1, timed(), f"{A.sell_padded() / s.nnz - 1:.1%}"))
        best = min(rows, key=lambda r: r[3])
        for r in rows:
            mark = " **" if r is best else ""
            print(f"| {s.name} (n={s.n}, nnz={s.nnz}) | {r[0]}{mark} | {r[1]} | {r[2]} | {r[3]:.1f} | {r[4]} | "
                  f"{alg / (r[3] * 1e-6) / 1e9:.0f} |")
        fmt, prm, us = A.tune()
        cs = A.get_sell() if fmt != FMT_CSR else ("", "")
        print(f"| {s.name} | tuner pick: {FORMAT_NAMES[fmt]}/{prm} | {cs[0]} | {cs[1]} | {us:.1f} | | "
              f"{alg / (us * 1e-6) / 1e9:.0f} |")
        del A, x, y
        plat.synchronize()


def solver_case(a, s, A, dt, fmt, prm, us, alg, sv):
    """Kernel times of the Jacobi sweep or the BiCGSTAB pass kernels."""
    plat = A.platform
    if a.solver == "jacobi":
        sol = lmp.Jacobi()
        sol.SetSolveMode(2)
        sol.SetNumIter(max(a.cg_iters, 1))
        names, extra = ["sweep"], [2 * s.n * sv]
    elif a.solver == "bicgstab":
        sol = lmp.BiCGSTAB()
        pc = lmp.PreconditionerBlockJacobiStand()
        pc.Init_Jacobi()
        sol.SetupPreconditioner(pc)
        names = ["spmv_q (A q, q.r0-type sums)", "s update", "spmv_s (A s, t.s, t.t)", "x/r update",
                 "direction"]
        extra = [s.n * sv, 5 * s.n * sv, s.n * sv, 8 * s.n * sv, 5 * s.n * sv]
    else:
        sol = lmp.GMRES()
        sol.InitParameter(a.basis, "RightPreconditioning")
        pc = lmp.PreconditionerBlockJacobiStand()
        pc.Init_Jacobi()
        sol.SetupPreconditioner(pc)
        names = ["cycle update", "restart", "spmv (A P v_j, w.V0)", "arnoldi step"]
        extra = [0, 0, s.n * sv, 0]
    sol.InitControl(100000, 0.0, 1e-12, 1e8)
    sol.SetupOperator(A)
    b = lmp.B200_lVector.from_numpy(s.b.astype(dt), platform=plat, dtype=dt)
    x0 = lmp.B200_lVector(s.n, platform=plat, dtype=dt)
    ms = sol.profile(b, x0, a.cg_iters)
    print(f"system n={s.n} nnz={s.nnz} dtype={a.dtype} schedule={FORMAT_NAMES[fmt]}/{prm} tuned_us={us:.1f}")
    for k, name in enumerate(names):
        nbytes = extra[k] + (alg if name.startswith(("sweep", "spmv")) else 0)
        if not nbytes:
            print(f"{a.solver} {name}: {ms[k]:.4f} ms")
            continue
        print(f"{a.solver} {name}: {ms[k]:.4f} ms, algorithmic {nbytes} bytes -> {nbytes / ms[k] / 1e6:.1f} GB/s")


BATCH3D_CELLS = (40, 50, 60, 70, 80, 90)  # --batch-dim 3: cells per axis, cycled


def batch_case(a):
    from .batch import Batch
    plat = lmp.init_platform(0)
    count = a.batch
    # the settings of bench.py's batch workload
    B = Batch(count, mixed=True, precond=True, rtol=1e-8, atol=0.0, dtol=1e8, inner_rtol=0.1, max_outer=60,
              tile_rows=a.tile_rows, index_bits=a.index_bits, platform=plat)
    if a.batch_dim == 3:
        # 3D Q1 systems (27 entries per row) of 41^3 .. 91^3 nodes, lognormal
        # kappa sigma 1, assembled on the device (the served stream's 3D kind)
        for i in range(count):
            B.add_q1(3, BATCH3D_CELLS[i % len(BATCH3D_CELLS)], 100 + i, 1.0)
        systems = list(range(count))
    else:
        systems = P.batch_systems(count, sigma=1.0, seed=P.SEED_BATCH)
        for s in systems:
            B.add_system(s)
    if a.items:
        B.set_items(*[int(v) for v in a.items.split(",")], adaptive=a.adaptive)
        print(f"item rows (K1, K2, K3) {B.items()}")
    else:
        rows, us = B.tune()
        if a.adaptive:
            B.set_items(*rows, adaptive=True)
        print(f"tuned item rows (K1, K2, K3) {rows}: pass {us:.1f} us")
    if a.profile_only:
        # launch order: K1 K2 K3 of the restart pass, then K1 K2 K3 per timed pass
        ms, nb = B.profile_pass(3)
        for name, t, b in zip(("K1 spmv+p.Ap", "K2 update", "K3 direction"), ms, nb):
            print(f"{name}: {t * 1e3:.1f} us, algorithmic {b} bytes -> {b / t / 1e6:.1f} GB/s")
        return
    for _ in range(a.solves):
        B.restart()
        t = time.perf_counter()
        passes = B.solve(a.chunk)
        dt = time.perf_counter() - t
        print(f"batch {len(systems)} systems tile_rows {a.tile_rows or 'default'} chunk {a.chunk} "
              f"adaptive {int(a.adaptive)}: "
              f"{passes} passes, {dt * 1e3:.1f} ms wall")


if __name__ == "__main__":
    main()
