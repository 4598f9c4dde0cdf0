"""Runs the C++ tests on the GPU:

* tests/cpp/test_lmp_adapter.cc: the reference's lmp/CG known answers through
  the C++ host layer ba_b200/host/b200_lmp.hpp;
* tests/cpp/test_hiflow_lmp.cc: HiFlow3's own lmp code (its CPU sources
  compiled unmodified into oracle/_ref: the lVector/lMatrix bases, the
  factories, lPreconditioner_Jacobi and the lmp cg()) running on the B200
  backend classes B200_lVector / B200_CSR_lMatrix (ba_b200/hiflow), against
  the reference's known answers and its own CPU runs.  The program is built
  where the HiFlow3 headers are (__graft_entry__.build) and runs prebuilt."""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


def test_cpp_host_layer():
    subprocess.run(["make", "-C", os.path.join(HERE, "cpp")], check=True, capture_output=True)
    p = subprocess.run([os.path.join(HERE, "cpp", "test_lmp_adapter")], capture_output=True, text=True,
                       timeout=300)
    assert p.returncode == 0, p.stdout + p.stderr
    assert p.stdout.strip().endswith("OK")


def test_hiflow_lmp_on_b200_classes():
    exe = os.path.join(HERE, "cpp", "test_hiflow_lmp")
    assert os.path.exists(exe), "tests/cpp/test_hiflow_lmp was not built (build() with the HiFlow3 tree present)"
    p = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    lines = [ln for ln in p.stdout.splitlines() if ln.startswith(("PASS", "FAIL"))]
    names = {ln.split()[1] for ln in lines}
    assert {"cg_test_known_answer", "lmp_test_spmv", "lmp_test_spmv_from_coo", "laplace_cg_f64",
            "laplace_cg_f64_jacobi", "laplace_cg_f32", "laplace_cg_f32_jacobi", "vector_dot_norm2", "vector_updates",
            "vector_casts", "matrix_nodiag_invdiag"} <= names, p.stdout
    assert p.returncode == 0 and not any(ln.startswith("FAIL") for ln in lines), p.stdout + p.stderr
