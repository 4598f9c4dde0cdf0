"""Runs the C++ host-layer test (tests/cpp/test_lmp_adapter.cc) on the GPU:
the reference's lmp/CG known answers through ba_b200/host/b200_lmp.hpp."""
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
