"""Records the reference's iteration counts (CG<LAD>, and BiCGSTAB<LAD> and
GMRES<LAD>(100) on the poisson3d matrix) on the full-size standard workloads
(tests/golden/workload_counts.json), by running HiFlow3's own lmp CPU classes
(oracle/_ref, NAIVE implementation, bit-identical to the C restatement) to
convergence here.  bench.py's CPU legs time a bounded sample
of iterations and scale it by these counts.

Usage (repository root, oracle/_ref built):  python tests/golden/make_workload_counts.py
"""
import json
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from ba_b200 import problems as P  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "workload_counts.json")


def main():
    out = {}
    if os.path.exists(OUT):
        out = json.load(open(OUT))
    for name, make, rtol in (("poisson3d_128", lambda: P.poisson_3d(128), 1e-10),
                             ("poisson2d_256", lambda: P.poisson_2d(256), 1e-10)):
        s = make()
        for precond in (True, False):
            key = f"{name}/{'jacobi' if precond else 'none'}/rtol{rtol:g}"
            if key in out:
                continue
            t = time.time()
            sysr = oracle.RefSystem(s.rowptr, s.col, s.val, impl=oracle.IMPL_NAIVE, nthreads=1)
            r, sec = sysr.cg(s.b, maxits=20000, atol=0.0, rtol=rtol, dtol=1e8, precond=precond)
            out[key] = {"iters": r.iters, "res": r.res, "res_init": r.res_init, "state": r.state,
                        "solve_seconds_1core": sec, "n": s.n, "nnz": s.nnz}
            print(key, out[key], f"{time.time() - t:.1f}s", flush=True)
            json.dump(out, open(OUT, "w"), indent=1)
    # BiCGSTAB<LAD> with right Jacobi preconditioning on the poisson3d matrix
    key = "poisson3d_128/bicgstab_jacobi/rtol1e-10"
    if key not in out:
        s = P.poisson_3d(128)
        t = time.time()
        r, restarts = oracle.ref_bicgstab(s.rowptr, s.col, s.val, s.b, maxits=20000, atol=0.0, rtol=1e-10,
                                          dtol=1e8, precond=True)
        out[key] = {"iters": r.iters, "restarts": restarts, "res": r.res, "res_init": r.res_init,
                    "state": r.state, "solve_seconds_1core": r.seconds, "n": s.n, "nnz": s.nnz}
        print(key, out[key], f"{time.time() - t:.1f}s", flush=True)
        json.dump(out, open(OUT, "w"), indent=1)
    # GMRES<LAD>(100) with right Jacobi preconditioning on the poisson3d matrix
    key = "poisson3d_128/gmres100_jacobi/rtol1e-10"
    if key not in out:
        s = P.poisson_3d(128)
        t = time.time()
        r = oracle.ref_gmres(s.rowptr, s.col, s.val, s.b, size_basis=100, maxits=20000, atol=0.0, rtol=1e-10,
                             dtol=1e8, precond=True)
        out[key] = {"iters": r.iters, "res": r.res, "res_init": r.res_init, "state": r.state,
                    "solve_seconds_1core": r.seconds, "n": s.n, "nnz": s.nnz}
        print(key, out[key], f"{time.time() - t:.1f}s", flush=True)
        json.dump(out, open(OUT, "w"), indent=1)


if __name__ == "__main__":
    main()
