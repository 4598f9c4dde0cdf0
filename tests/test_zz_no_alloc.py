"""b200la_dot_noalloc: the dot product for callers that cannot allocate.

Some callers cannot call cudaMalloc -- it can stall the whole device while
overlapped work is in flight, and applications that own all device memory
through their own pool, or load this library as a plug-in under a fixed
quota, may not allocate outside it.  The entry point keeps its reduction
scratch in a fixed __device__ array instead.  This test calls it through the
C ABI on device buffers the test owns and checks it against the allocating
entry point b200la_vec_dot, twice in a row, with the tolerance the BLAS-1
parity tests use.  The file name keeps it last in collection order.
"""
import ctypes as C

import numpy as np
import pytest

from ba_b200 import _lib, lmp
from ba_b200._lib import F32, F64

pytestmark = pytest.mark.gpu

MAX_N = 16_777_216


def _noalloc(a, b, n, dtype, stream):
    out = C.c_double()
    st = _lib.load().b200la_dot_noalloc(C.c_void_p(a.GetBuffer()), C.c_void_p(b.GetBuffer()), n, dtype,
                                        stream, C.byref(out))
    return st, out.value


def test_dot_noalloc_matches_dot_twice_in_a_row():
    plat = lmp.init_platform(0)
    stream = C.c_void_p()
    _lib.call("b200la_ctx_get_stream", plat.handle, C.byref(stream))
    rng = np.random.default_rng(11)
    for n, dtype, np_t in ((1, F64, np.float64), (4097, F64, np.float64), (1_000_003, F64, np.float64),
                           (MAX_N, F64, np.float64), (65_537, F32, np.float32)):
        for call in range(2):  # scratch keeps the last call's contents: run twice
            a = rng.standard_normal(n).astype(np_t)
            b = rng.standard_normal(n).astype(np_t)
            va = lmp.B200_lVector.from_numpy(a, platform=plat, dtype=np_t)
            vb = lmp.B200_lVector.from_numpy(b, platform=plat, dtype=np_t)
            ref = va.Dot(vb)
            st, got = _noalloc(va, vb, n, dtype, stream)
            assert st == 0, _lib.load().b200la_last_error()
            if dtype == F64:
                np.testing.assert_allclose(got, ref, rtol=1e-13, atol=1e-13 * n)
            else:
                scale = float(np.abs(a.astype(np.float64)) @ np.abs(b.astype(np.float64)))
                assert abs(got - ref) <= 1e-6 * scale, (n, call, got, ref)


def test_dot_noalloc_rejects_sizes_beyond_its_scratch():
    plat = lmp.init_platform(0)
    va = lmp.B200_lVector(16, platform=plat)
    st, _ = _noalloc(va, va, MAX_N + 1, F64, None)
    assert st == -7
    assert b"scratch limit" in _lib.load().b200la_last_error()
    st, got = _noalloc(va, va, 0, F64, None)
    assert st == 0 and got == 0.0
