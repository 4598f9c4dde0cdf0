"""Request loop for PCG solves (no counterpart in the reference, which solves
one system per CG<LAD> call).

``Server`` wraps the b200la_server_* C ABI: a worker thread in the library
admits queued solves into the slots of one batch while the resident systems'
device bytes fit the HBM budget, advances every resident system with chunked
CUDA-graph launches, and harvests finished systems (solution and result
copied to the host, slot freed).  Requests that arrive while others are on
the GPU join the next launch (continuous batching).

Adaptive work items are on by default here: a served stream often ends with
a few large systems running alone, where smaller items keep every warp busy
(measured +4% solves/s on the seeded stream, -1% on a full fixed batch).
"""
from __future__ import annotations

import ctypes as C
import sys
import time

import numpy as np

from ._lib import BatchParams, ServerParams, ServerStats, SysResult, call, load
from .batch import SystemResult
from .lmp import Platform, _finalizing, init_platform


class Server:
    def __init__(self, capacity: int = 256, *, mixed: bool = True, precond: bool = True, rtol: float = 1e-8,
                 atol: float = 0.0, dtol: float = 1e8, inner_rtol: float = 0.1, max_outer: int = 30,
                 inner_maxits: int = 100000, tile_rows: int = 0, hbm_budget: int = 0, chunk_passes: int = 32,
                 max_skips: int = 8, adaptive: bool = True, restart_inner: bool = False,
                 platform: Platform | None = None):
        self.platform = platform or init_platform()
        bp = BatchParams(int(capacity), int(mixed), int(precond), int(max_outer), int(inner_maxits), int(adaptive),
                         int(tile_rows), 0, float(atol), float(rtol), float(dtol), float(inner_rtol),
                         1 if restart_inner else 0)
        prm = ServerParams(bp, int(hbm_budget), int(chunk_passes), int(max_skips))
        self.handle = C.c_void_p()
        call("b200la_server_start", self.platform.handle, C.byref(prm), C.byref(self.handle))
        self._n = {}

    # ---- submission
    def submit(self, rowptr, col, val, rhs, x0=None) -> int:
        """Queue a host CSR system (copied at submission); returns its id."""
        rp = np.ascontiguousarray(rowptr, np.int32)
        cl = np.ascontiguousarray(col, np.int32)
        vv = np.ascontiguousarray(val, np.float64)
        bb = np.ascontiguousarray(rhs, np.float64)
        xx = None if x0 is None else np.ascontiguousarray(x0, np.float64)
        rid = C.c_int64()
        call("b200la_server_submit_csr", self.handle, rp.shape[0] - 1, cl.shape[0],
             rp.ctypes.data_as(C.c_void_p), cl.ctypes.data_as(C.c_void_p), vv.ctypes.data_as(C.c_void_p),
             bb.ctypes.data_as(C.c_void_p), None if xx is None else xx.ctypes.data_as(C.c_void_p),
             C.byref(rid))
        self._n[rid.value] = rp.shape[0] - 1
        return rid.value

    def submit_system(self, s, x0=None) -> int:
        return self.submit(s.rowptr, s.col, s.val, s.b, x0)

    def submit_q1(self, dim: int, cells: int, seed: int, sigma: float) -> int:
        """Queue a Q1 diffusion system that the device assembles at admission."""
        rid = C.c_int64()
        call("b200la_server_submit_q1", self.handle, int(dim), int(cells), C.c_uint64(seed), float(sigma),
             C.byref(rid))
        self._n[rid.value] = (cells + 1) ** dim
        return rid.value

    # ---- results
    def poll(self, rid: int, with_x: bool = True):
        """None while queued or running, else (SystemResult, latency ms)."""
        done, lat, r = C.c_int(), C.c_double(), SysResult()
        n = self._n.get(rid)
        x = np.empty(n, np.float64) if (with_x and n is not None) else None
        call("b200la_server_poll", self.handle, int(rid), C.byref(done),
             None if x is None else x.ctypes.data_as(C.c_void_p), C.byref(r), C.byref(lat))
        if not done.value:
            return None
        res = SystemResult(r.state, r.solver_state, r.iters, r.outer, bool(r.phase_done), r.res, r.res_init,
                           r.res_rel, r.device_us, x)
        return res, lat.value

    def wait(self, rid: int, timeout: float = 600.0, with_x: bool = True):
        done = C.c_int()
        deadline = time.monotonic() + timeout
        while True:
            left = deadline - time.monotonic()
            call("b200la_server_wait", self.handle, int(rid), max(min(left, 1.0), 0.0), C.byref(done))
            if done.value:
                return self.poll(rid, with_x)
            if left <= 0:
                raise TimeoutError(f"request {rid} not done after {timeout} s")

    def release(self, rid: int):
        call("b200la_server_release", self.handle, int(rid))
        self._n.pop(rid, None)

    def drain(self, timeout: float = 600.0):
        call("b200la_server_drain", self.handle, float(timeout))

    def stats(self) -> dict:
        st = ServerStats()
        call("b200la_server_get_stats", self.handle, C.byref(st))
        return {k: getattr(st, k) for k, _ in ServerStats._fields_}

    def reset_stats(self):
        call("b200la_server_reset_stats", self.handle)

    def close(self):
        if self.handle:
            load().b200la_server_stop(self.handle)
            self.handle = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self, _fin=_finalizing):  # bound at definition: globals are gone at exit
        if _fin():
            return
        try:
            self.close()
        except Exception:
            pass
