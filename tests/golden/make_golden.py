"""Regenerates tests/golden/*.json from the reference's own compiled code.

Runs HiFlow3's lmp CPU sources, built by oracle/ref/Makefile into
oracle/_ref/libhiflow_lmp_ref.so, on the small systems below and records
their iteration counts, residuals and solutions.  The known answers of the
reference's own unit tests are recorded beside them, verbatim from:
  tests/cg_test.cc:92-94     x = (-0.25, -1.5, -0.75) for cg() on the 3x3 stencil
  tests/lmp_test.cc:80-82    A*(1,-2,0) = (4,-5,2) (7-nnz CSR)
  tests/cuda_test.cc:76-78   A*(1.2,-2.3,0.7) = (4.7,-6.5,3.7) (dense-stored 3x3)
and the reference's Jacobi<LAD>, BiCGSTAB<LAD> and GMRES<LAD> (restated over
the same compiled objects) on further systems, in reference_krylov_runs.json.

Usage (from the repository root, where oracle/_ref exists):
    python tests/golden/make_golden.py
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from ba_b200 import problems as P  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def cases():
    yield P.poisson_2d(16)
    yield P.poisson_2d(64)
    yield P.q1_system(2, 33, 11, 1.0, "varcoef2d_33_s1")
    yield P.q1_system(3, 8, 12, 0.0, "poisson3d_8")
    yield P.q1_system(3, 12, 13, 2.0, "varcoef3d_12_s2")
    yield P.random_spd(17, 1, empty_rows=0)
    yield P.random_spd(33, 2, empty_rows=3)
    yield P.random_spd(257, 3, density=0.02, empty_rows=5)


def main():
    if not oracle.ref_available():
        raise SystemExit("oracle/_ref not built: run `make -C oracle` first")
    known = {
        "cg_test_3x3": {"source": "tests/cg_test.cc:92-94", "x": [-0.25, -1.5, -0.75]},
        "lmp_test_spmv": {"source": "tests/lmp_test.cc:80-82", "x": [1.0, -2.0, 0.0],
                          "y": [4.0, -5.0, 2.0]},
        "cuda_test_spmv": {"source": "tests/cuda_test.cc:76-78", "x": [1.2, -2.3, 0.7],
                           "y": [4.7, -6.5, 3.7], "tol": 1e-12},
    }
    solves = []
    for s in cases():
        entry = {"name": s.name, "n": s.n, "nnz": s.nnz, "sha_rowptr": sha(s.rowptr),
                 "sha_col": sha(s.col), "sha_val": sha(s.val), "sha_b": sha(s.b), "runs": []}
        for dtype, rtol in (("f64", 1e-10), ("f32", 1e-5)):
            for precond in (False, True):
                dt = np.float64 if dtype == "f64" else np.float32
                r = oracle.ref_cg(s.rowptr, s.col, s.val, s.b, maxits=20000, atol=0.0, rtol=rtol,
                                  dtol=1e8, precond=precond, dtype=dt)
                entry["runs"].append({
                    "dtype": dtype, "precond": precond, "rtol": rtol, "iters": r.iters,
                    "res": r.res, "res_init": r.res_init, "state": r.state,
                    "x": [float(v) for v in r.x], "sha_x": sha(r.x)})
        lr = oracle.ref_lmp_cg(s.rowptr, s.col, s.val, s.b, rel_eps=1e-10, abs_eps=0.0,
                               max_iter=20000)
        entry["lmp_cg"] = {"rel_eps": 1e-10, "max_iter_out": lr.iters, "sha_x": sha(lr.x)}
        xs = P.uniform01(99, s.n, stream=5)
        entry["spmv"] = {"x_seed": 99, "x_stream": 5,
                         "y": [float(v) for v in oracle.ref_spmv(s.rowptr, s.col, s.val, xs)]}
        if s.n > 300:
            for run in entry["runs"]:
                run.pop("x")
            entry["spmv"].pop("y")
            entry["spmv"]["sha_y"] = sha(oracle.ref_spmv(s.rowptr, s.col, s.val, xs))
        solves.append(entry)
    with open(os.path.join(OUT, "reference_known_answers.json"), "w") as f:
        json.dump(known, f, indent=1)
    with open(os.path.join(OUT, "reference_cg_runs.json"), "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py", "cases": solves}, f)
    print("wrote", len(solves), "cases")
    krylov_runs()


# TransformFromCOO cases: (rows, cols, triplets, seed); duplicates, empty rows
COO_CASES = ((50, 60, 400, 1), (300, 300, 5000, 2), (1000, 800, 3000, 3))


def coo_triplets(nrow, ncol, nnz, seed):
    """Seeded random triplets in random order, with duplicate positions."""
    rng = np.random.default_rng(seed)
    return (rng.integers(0, nrow, nnz).astype(np.int32), rng.integers(0, ncol, nnz).astype(np.int32),
            rng.standard_normal(nnz))


# GMRES<LAD> restart lengths (basis sizes)
GMRES_BASIS = (10, 30, 100)
# Jacobi<LAD> runs: (mode, w, inner_iter, smooth_iter, maxits)
JACOBI_RUNS = ((0, 1.0, 1, 1, 20000), (1, 0.7, 3, 1, 20000), (2, 1.0, 2, 7, 20000), (3, 0.6, 2, 1, 5))


def krylov_cases():
    yield P.poisson_2d(16)
    yield P.q1_system(2, 33, 11, 1.0, "varcoef2d_33_s1")
    yield P.convdiff_2d(24, 20.0)
    yield P.convdiff_2d(16, 200.0)
    yield P.q1_system(3, 8, 12, 0.0, "poisson3d_8")
    yield P.random_spd(33, 2, empty_rows=3)


def krylov_runs():
    """Jacobi<LAD>, BiCGSTAB<LAD> and GMRES<LAD> restated over the compiled lmp
    objects (oracle/ref/ref_driver.cc) -> reference_krylov_runs.json."""
    out = []
    for s in krylov_cases():
        entry = {"name": s.name, "n": s.n, "nnz": s.nnz, "sha_val": sha(s.val), "sha_b": sha(s.b),
                 "jacobi": [], "bicgstab": []}
        for mode, w, inner, smooth, maxits in JACOBI_RUNS:
            r = oracle.ref_jacobi(s.rowptr, s.col, s.val, s.b, mode=mode, maxits=maxits, inner_iter=inner,
                                  smooth_iter=smooth, w=w, atol=0.0, rtol=1e-6, dtol=1e8)
            run = {"mode": mode, "w": w, "inner_iter": inner, "smooth_iter": smooth, "maxits": maxits,
                   "rtol": 1e-6, "iters": r.iters, "state": r.state, "res": r.res,
                   "res_init": r.res_init, "sha_x": sha(r.x)}
            if s.n <= 300:
                run["x"] = [float(v) for v in r.x]
            entry["jacobi"].append(run)
        for precond in (False, True):
            r, restarts = oracle.ref_bicgstab(s.rowptr, s.col, s.val, s.b, maxits=5000, atol=0.0,
                                              rtol=1e-10, dtol=1e8, precond=precond)
            run = {"precond": precond, "rtol": 1e-10, "maxits": 5000, "iters": r.iters, "state": r.state,
                   "restarts": restarts, "res": r.res, "res_init": r.res_init, "sha_x": sha(r.x)}
            if s.n <= 300:
                run["x"] = [float(v) for v in r.x]
            entry["bicgstab"].append(run)
        entry["gmres"] = []
        for precond in (False, True):
            for m in GMRES_BASIS:
                r = oracle.ref_gmres(s.rowptr, s.col, s.val, s.b, size_basis=m, maxits=3000, atol=0.0,
                                     rtol=1e-10, dtol=1e8, precond=precond)
                run = {"precond": precond, "size_basis": m, "rtol": 1e-10, "maxits": 3000, "iters": r.iters,
                       "state": r.state, "res": r.res, "res_init": r.res_init, "sha_x": sha(r.x)}
                if s.n <= 300:
                    run["x"] = [float(v) for v in r.x]
                entry["gmres"].append(run)
        out.append(entry)
    coo = []
    for nrow, ncol, nnz, seed in COO_CASES:
        rows, cols, vals = coo_triplets(nrow, ncol, nnz, seed)
        rp, c, v = oracle.ref_coo_to_csr(nrow, ncol, rows, cols, vals)
        coo.append({"nrow": nrow, "ncol": ncol, "nnz": nnz, "seed": seed, "sha_rowptr": sha(rp),
                    "sha_col": sha(c), "sha_val": sha(v)})
    with open(os.path.join(OUT, "reference_krylov_runs.json"), "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py", "cases": out, "coo_to_csr": coo}, f)
    print("wrote", len(out), "Jacobi/BiCGSTAB/GMRES cases")


if __name__ == "__main__":
    main()
