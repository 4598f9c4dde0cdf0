"""Records the reference's solutions of the full-size workloads as
fingerprints (tests/golden/reference_fullsize_solutions.json): HiFlow3's own
lmp CPU classes (oracle/_ref, NAIVE implementation, one thread -- the exact
CG<LAD> iteration counts) solve

* poisson3d_128 (the 3D Q1 Poisson workload, 128^3 cells) and
  varcoef3d_128 (the same grid with a lognormal coefficient, sigma = 2) by FP64
  Jacobi-PCG to rel. 1e-10 (the iteration count and solution the device's
  FP64 solve is held to) and to rel. 1e-13 (the FP64 CPU CG oracle that
  mixed-precision results state their error against);
* a fixed stratified sample of 32 systems of the 1,024-system batch
  workload (rank 0's seed) by FP64 Jacobi-PCG to rel. 1e-12 (the oracle of
  the batch's error statement).

A solution is stored as problems.solution_probe(x): its norm, 64 Rademacher
projections and 2,048 sampled entries (a 17 MB vector would not belong in the
repository); problems.probe_error() turns two fingerprints into an error.

Usage (repository root, oracle/_ref built):
    python tests/golden/make_fullsize_solutions.py   (a few minutes, one process per job)
"""
import json
import multiprocessing as mp
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_fullsize_solutions.json")
BATCH_SAMPLE = 32


def _solve(job):
    import oracle
    from ba_b200 import problems as P
    name, rtol = job
    t = time.time()
    if name == "batch1024_sample":
        systems = P.batch_systems(1024, sigma=1.0, seed=P.SEED_BATCH)
        pick = P.stratified_sample([s.nnz for s in systems], BATCH_SAMPLE)
        out = {}
        for i in pick:
            s = systems[i]
            r = oracle.ref_cg(s.rowptr, s.col, s.val, s.b, maxits=100000, atol=0.0, rtol=rtol, dtol=1e8,
                              precond=True, impl=oracle.IMPL_NAIVE, nthreads=1)
            out[str(i)] = {"name": s.name, "iters": r.iters, "res": r.res, "res_init": r.res_init,
                           "state": r.state, "n": s.n, "nnz": s.nnz, "probe": P.solution_probe(r.x)}
        return f"{name}/jacobi/rtol{rtol:g}", {"systems": out, "indices": pick, "seconds": time.time() - t}
    s = P.poisson_3d(128) if name == "poisson3d_128" else P.varcoef_3d(128, 2.0)
    sysr = oracle.RefSystem(s.rowptr, s.col, s.val, impl=oracle.IMPL_NAIVE, nthreads=1)
    r, sec = sysr.cg(s.b, maxits=20000, atol=0.0, rtol=rtol, dtol=1e8, precond=True)
    sysr.close()
    return f"{name}/jacobi/rtol{rtol:g}", {"iters": r.iters, "res": r.res, "res_init": r.res_init,
                                           "state": r.state, "n": s.n, "nnz": s.nnz,
                                           "solve_seconds_1core": sec, "probe": P.solution_probe(r.x)}


def main():
    out = json.load(open(OUT)) if os.path.exists(OUT) else {}
    jobs = [("poisson3d_128", 1e-10), ("poisson3d_128", 1e-13), ("varcoef3d_128", 1e-10),
            ("varcoef3d_128", 1e-13), ("batch1024_sample", 1e-12)]
    jobs = [j for j in jobs if f"{j[0]}/jacobi/rtol{j[1]:g}" not in out]
    with mp.get_context("spawn").Pool(len(jobs) or 1) as pool:
        for key, rec in pool.imap_unordered(_solve, jobs):
            out[key] = rec
            print(key, {k: v for k, v in rec.items() if k not in ("probe", "systems")}, flush=True)
            json.dump(out, open(OUT, "w"), indent=0)


if __name__ == "__main__":
    main()
