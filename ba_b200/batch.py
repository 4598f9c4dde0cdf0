"""Batched and served PCG over many independent systems (no counterpart in
the reference, which solves one system per CG<LAD> call).

``Batch`` wraps the b200la_batch_* C ABI: systems are uploaded into slots,
``run`` advances every running system with one CUDA-graph launch, and
systems can be added and removed between runs (continuous batching).
"""
from __future__ import annotations

import ctypes as C
import sys
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import BatchParams, SysResult, call, load
from .lmp import Platform, _finalizing, init_platform


@dataclass
class SystemResult:
    state: int
    solver_state: int
    iters: int
    outer: int
    done: bool
    res: float
    res_init: float
    res_rel: float
    device_us: float
    x: np.ndarray | None = None


def slot_bytes(n: int, nnz: int, max_row: int, mixed: bool) -> int:
    out = C.c_int64()
    call("b200la_batch_slot_bytes", int(n), int(nnz), int(max_row), 1 if mixed else 0, C.byref(out))
    return out.value


class Batch:
    def __init__(self, capacity: int, *, mixed: bool = True, precond: bool = True, rtol: float = 1e-8,
                 atol: float = 0.0, dtol: float = 1e8, inner_rtol: float = 0.1, max_outer: int = 30,
                 inner_maxits: int = 100000, adaptive: bool = False, tile_rows: int = 0, index_bits: int = 0,
                 restart_inner: bool = False, platform: Platform | None = None):
        """Mixed mode: each FP32 inner pass ends once its residual has fallen
        by inner_rtol; the FP64 residual then replaces it and the inner PCG
        goes on with its search direction (restart_inner=True restarts it
        from p = z each pass instead, as MPIR does; give it a tighter
        inner_rtol such as 1e-4)."""
        self.platform = platform or init_platform()
        self.mixed = mixed
        prm = BatchParams(int(capacity), int(mixed), int(precond), int(max_outer), int(inner_maxits),
                          int(adaptive), int(tile_rows), int(index_bits), float(atol), float(rtol), float(dtol),
                          float(inner_rtol), 1 if restart_inner else 0)
        self.handle = C.c_void_p()
        call("b200la_batch_create", self.platform.handle, C.byref(prm), C.byref(self.handle))
        self._keep = {}
        self._sizes = {}
        self._outs = {}  # registered output arrays, kept alive until read

    def add(self, rowptr, col, val, rhs, x0=None) -> int:
        rp = np.ascontiguousarray(rowptr, np.int32)
        cl = np.ascontiguousarray(col, np.int32)
        vv = np.ascontiguousarray(val, np.float64)
        bb = np.ascontiguousarray(rhs, np.float64)
        xx = None if x0 is None else np.ascontiguousarray(x0, np.float64)
        slot = C.c_int()
        call("b200la_batch_add", self.handle, rp.shape[0] - 1, cl.shape[0], rp.ctypes.data_as(C.c_void_p),
             cl.ctypes.data_as(C.c_void_p), vv.ctypes.data_as(C.c_void_p), bb.ctypes.data_as(C.c_void_p),
             None if xx is None else xx.ctypes.data_as(C.c_void_p), C.byref(slot))
        # host buffers must stay valid until the copies run (next run)
        self._keep[slot.value] = (rp, cl, vv, bb, xx)
        self._sizes[slot.value] = rp.shape[0] - 1
        return slot.value

    def add_many(self, systems) -> list[int]:
        """Add many systems, each (rowptr, col, val, rhs[, x0]), with one wait
        for all the device checks; raises on the first failure (the others
        that succeeded stay added: see `last_slots` and `last_status`)."""
        arrs = []
        for t in systems:
            rp = np.ascontiguousarray(t[0], np.int32)
            cl = np.ascontiguousarray(t[1], np.int32)
            vv = np.ascontiguousarray(t[2], np.float64)
            bb = np.ascontiguousarray(t[3], np.float64)
            xx = None if len(t) < 5 or t[4] is None else np.ascontiguousarray(t[4], np.float64)
            arrs.append((rp, cl, vv, bb, xx))
        k = len(arrs)
        ptr = lambda a: None if a is None else a.ctypes.data  # noqa: E731
        n = (C.c_int * k)(*[a[0].shape[0] - 1 for a in arrs])
        nnz = (C.c_int64 * k)(*[a[1].shape[0] for a in arrs])
        P = C.c_void_p * k
        slots, status = (C.c_int * k)(), (C.c_int * k)()
        rc = load().b200la_batch_add_many(self.handle, k, n, nnz, P(*[ptr(a[0]) for a in arrs]),
                                          P(*[ptr(a[1]) for a in arrs]), P(*[ptr(a[2]) for a in arrs]),
                                          P(*[ptr(a[3]) for a in arrs]), P(*[ptr(a[4]) for a in arrs]), slots, status)
        out = list(slots)
        for j, sl in enumerate(out):
            if sl >= 0:
                self._sizes[sl] = arrs[j][0].shape[0] - 1
        self.last_status = list(status)
        self.last_slots = out
        _lib.check(rc)
        return out

    def add_system(self, s, x0=None) -> int:
        return self.add(s.rowptr, s.col, s.val, s.b, x0)

    def add_q1(self, dim: int, cells: int, seed: int, sigma: float) -> int:
        """Assemble a Q1 diffusion system on the device into a free slot."""
        slot = C.c_int()
        call("b200la_batch_add_q1", self.handle, int(dim), int(cells), C.c_uint64(seed), float(sigma),
             C.byref(slot))
        n, nnz = C.c_int(), C.c_int64()
        call("b200la_batch_slot_size", self.handle, slot.value, C.byref(n), C.byref(nnz))
        self._sizes[slot.value] = n.value
        return slot.value

    def get_system(self, slot: int):
        """(rowptr, col, val, rhs) of a slot, copied back to the host."""
        n, nnz = C.c_int(), C.c_int64()
        call("b200la_batch_slot_size", self.handle, int(slot), C.byref(n), C.byref(nnz))
        rp = np.empty(n.value + 1, np.int32)
        cl = np.empty(nnz.value, np.int32)
        vv = np.empty(nnz.value, np.float64)
        bb = np.empty(n.value, np.float64)
        call("b200la_batch_get_system", self.handle, int(slot), rp.ctypes.data_as(C.c_void_p),
             cl.ctypes.data_as(C.c_void_p), vv.ctypes.data_as(C.c_void_p), bb.ctypes.data_as(C.c_void_p))
        return rp, cl, vv, bb

    def remove(self, slot: int):
        call("b200la_batch_remove", self.handle, int(slot))
        self._keep.pop(slot, None)
        self._sizes.pop(slot, None)
        self._outs.pop(slot, None)

    def remove_many(self, slots):
        """Free many slots with one call (all in use and distinct, else none is freed)."""
        slots = [int(s) for s in slots]
        k = len(slots)
        call("b200la_batch_remove_many", self.handle, k, (C.c_int * k)(*slots))
        for s in slots:
            self._keep.pop(s, None)
            self._sizes.pop(s, None)
            self._outs.pop(s, None)

    def run(self, max_passes: int = 1 << 30) -> int:
        active = C.c_int()
        call("b200la_batch_run", self.handle, int(max_passes), C.byref(active))
        self._keep.clear()
        return active.value

    def result(self, slot: int, with_x: bool = True) -> SystemResult:
        r = SysResult()
        x = None
        ptr = None
        if with_x:
            x = np.empty(self.slot_n(slot), np.float64)
            ptr = x.ctypes.data_as(C.c_void_p)
        call("b200la_batch_result", self.handle, int(slot), ptr, C.byref(r))
        if with_x:
            self._outs.pop(int(slot), None)
        return SystemResult(r.state, r.solver_state, r.iters, r.outer, bool(r.phase_done), r.res, r.res_init,
                            r.res_rel, r.device_us, x)

    def set_outputs(self, slots, arrays):
        """Register float64 host arrays (contiguous, at least n elements; pinned
        ones keep the copies asynchronous) to receive the slots' solutions as
        soon as runs see them finished, overlapping the passes still running;
        `results(slots, out=arrays)` then only waits for those copies.  The
        arrays are kept alive here until the results are read."""
        slots = [int(s) for s in slots]
        arrays = list(arrays)
        if len(arrays) != len(slots):
            raise _lib.B200LAError(-1, "set_outputs: one array per slot")
        for s, a in zip(slots, arrays):
            n = self._sizes.get(s)
            if n is None or a.dtype != np.float64 or not a.flags.c_contiguous or a.size < n:
                raise _lib.B200LAError(-1, f"set_outputs: slot {s} needs a contiguous float64 array of {n}")
        k = len(slots)
        call("b200la_batch_set_outputs", self.handle, k, (C.c_int * k)(*slots),
             (C.c_void_p * k)(*[a.ctypes.data for a in arrays]))
        for s, a in zip(slots, arrays):
            self._outs[s] = a

    def results(self, slots, with_x: bool = True, out=None) -> list[SystemResult]:
        """Results of many slots with one wait for all the solution copies;
        `out` may give preallocated float64 arrays (e.g. pinned) per slot."""
        slots = [int(s) for s in slots]
        k = len(slots)
        rs = (SysResult * k)()
        sl = (C.c_int * k)(*slots)
        xs = None
        ptrs = None
        if with_x:
            xs = list(out) if out is not None else [np.empty(self.slot_n(s), np.float64) for s in slots]
            ptrs = (C.c_void_p * k)(*[x.ctypes.data for x in xs])
        call("b200la_batch_results", self.handle, k, sl, ptrs, rs)
        if with_x:
            for sl_ in slots:
                self._outs.pop(sl_, None)  # registrations end with a read of x
        return [SystemResult(r.state, r.solver_state, r.iters, r.outer, bool(r.phase_done), r.res, r.res_init,
                             r.res_rel, r.device_us, None if xs is None else xs[j]) for j, r in enumerate(rs)]

    def slot_n(self, slot: int) -> int:
        return self._sizes[slot]

    def launch(self, max_passes: int = 64):
        """Start up to max_passes passes over the running systems and return at
        once; adds made meanwhile overlap the launch and join the next one."""
        call("b200la_batch_launch", self.handle, int(max_passes))

    def solve(self, chunk_passes: int = 64) -> int:
        """Run until every system has finished, compacting the tile list every
        chunk_passes passes; returns the passes taken."""
        n = C.c_int()
        call("b200la_batch_solve", self.handle, int(chunk_passes), C.byref(n))
        self._keep.clear()
        return n.value

    def last_passes(self) -> int:
        """Device-loop passes taken by the last run (each pass = 3 kernel launches)."""
        n = C.c_int()
        call("b200la_batch_last_run", self.handle, C.byref(n), None)
        return n.value

    def restart(self):
        """Restart every system from x = 0 (matrices and right-hand sides stay resident)."""
        call("b200la_batch_restart", self.handle)
        self._outs.clear()

    def tune(self) -> tuple[tuple[int, int, int], float]:
        """Pick the warp item sizes (rows) of K1 (SpMV), K2 (update) and K3
        (direction) by timing real passes (every system's state is
        restored); returns ((k1, k2, k3), microseconds per pass)."""
        rows, us = (C.c_int * 3)(), C.c_double()
        call("b200la_batch_tune", self.handle, rows, C.byref(us))
        return tuple(rows), us.value

    def set_items(self, k1: int, k2: int, k3: int, adaptive: bool = True):
        """Set the item sizes (rows, multiples of 32) of K1, K2, K3; with
        adaptive, lightly loaded runs use smaller items."""
        call("b200la_batch_set_items", self.handle, int(k1), int(k2), int(k3), int(adaptive))

    def items(self) -> tuple[int, int, int]:
        rows = (C.c_int * 3)()
        call("b200la_batch_get_items", self.handle, rows)
        return tuple(rows)

    def profile_pass(self, reps: int = 5) -> tuple[list[float], list[int]]:
        """Per-kernel ms of an inner pass (K1 SpMV + p.Ap, K2 update, K3
        direction) and each kernel's algorithmic bytes.  Restarts every system."""
        ms = (C.c_double * 3)()
        nb = (C.c_int64 * 3)()
        call("b200la_batch_profile_pass", self.handle, int(reps), ms, nb)
        return list(ms), list(nb)

    def profile(self, reps: int = 5) -> tuple[float, int]:
        """(ms per batched SpMV over every slot, its algorithmic bytes)."""
        ms, nb = C.c_double(), C.c_int64()
        call("b200la_batch_profile", self.handle, int(reps), C.byref(ms), C.byref(nb))
        return ms.value, nb.value

    def info(self) -> tuple[int, int]:
        u, b = C.c_int(), C.c_int64()
        call("b200la_batch_info", self.handle, C.byref(u), C.byref(b))
        return u.value, b.value

    def close(self):
        if self.handle:
            load().b200la_batch_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self, _fin=_finalizing):  # bound at definition: globals are gone at exit
        if _fin():
            return
        try:
            self.close()
        except Exception:
            pass
