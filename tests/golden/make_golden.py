"""Regenerates tests/golden/*.json from the reference's own compiled code.

Runs HiFlow3's lmp CPU sources, built by oracle/ref/Makefile into
oracle/_ref/libhiflow_lmp_ref.so, on the small systems below and records
their iteration counts, residuals and solutions.  The known answers of the
reference's own unit tests are recorded beside them, verbatim from:
  tests/cg_test.cc:92-94     x = (-0.25, -1.5, -0.75) for cg() on the 3x3 stencil
  tests/lmp_test.cc:80-82    A*(1,-2,0) = (4,-5,2) (7-nnz CSR)
  tests/cuda_test.cc:76-78   A*(1.2,-2.3,0.7) = (4.7,-6.5,3.7) (dense-stored 3x3)

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


if __name__ == "__main__":
    main()
