"""Host-side mirror of HiFlow3's lmp / linear_solver interface for the PCG path.

The classes keep the reference's names, argument meaning and results so code
written against lmp reads the same:

* ``init_platform``            ~ init_platform_gpu   (lmp/cuda/platform_management_gpu.cu:78)
* ``B200_lVector``             ~ lVector<T>          (lmp/lvector.h:38-321)
* ``B200_CSR_lMatrix``         ~ CSR_lMatrix<T>      (lmp/lmatrix.h:39-468)
* ``init_vector / init_matrix``~ the factories       (lmp/init_vec_mat.cc:146, :259)
* ``IterateControl``           ~ common/iterate_control.h
* ``PreconditionerBlockJacobiStand`` with ``Init_Jacobi``
                               ~ linear_solver/preconditioner_bjacobi_standard.cc:77-196
* ``CG``                       ~ CG<LAD> (linear_solver/cg.h:39-247): InitControl,
  SetupOperator, SetupPreconditioner, Solve -> LinearSolverState, iter(), res()

Differences: errors raise B200LAError instead of exit(-1); all compute runs in
libb200la.so on the GPU (no CPU fallback).
"""
from __future__ import annotations

import ctypes as C
import sys

import numpy as np

from . import _lib
from ._lib import F32, F64, FMT_CSR, FMT_SELL, B200LAError, CgParams, CgResult, call, load

kSolverSuccess, kSolverExceeded, kSolverError = 0, 1, 2
_finalizing = sys.is_finalizing  # held: sys may be torn down before __del__ runs at exit

_NP = {F64: np.float64, F32: np.float32}


def _dt(dtype) -> int:
    if dtype in (F64, F32):
        return dtype
    d = np.dtype(dtype)
    if d == np.float64:
        return F64
    if d == np.float32:
        return F32
    raise TypeError(f"unsupported dtype {dtype}")


class Platform:
    """A device context (one stream, reduction scratch)."""

    def __init__(self, device: int = 0):
        self.handle = C.c_void_p()
        call("b200la_ctx_create", device, C.byref(self.handle))
        self.device = device

    def synchronize(self):
        call("b200la_ctx_synchronize", self.handle)

    def set_stream(self, stream_ptr: int | None):
        call("b200la_ctx_set_stream", self.handle, C.c_void_p(stream_ptr or 0))

    def set_graphs(self, on: bool):
        """Run device loops as CUDA-graph WHILE nodes (default) or, with
        False, launch the same kernels one by one from a host loop."""
        call("b200la_ctx_set_graphs", self.handle, 1 if on else 0)

    @property
    def num_sms(self) -> int:
        n = C.c_int()
        call("b200la_ctx_num_sms", self.handle, C.byref(n))
        return n.value

    def close(self):
        if self.handle:
            load().b200la_ctx_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self, _fin=_finalizing):  # bound at definition: globals are gone at exit
        # at interpreter exit the process teardown releases device memory;
        # destroying contexts in arbitrary finalization order is unsafe
        if _fin():
            return
        try:
            self.close()
        except Exception:
            pass


_default = None


def init_platform(device: int = 0) -> Platform:
    global _default
    if _default is None:
        _default = Platform(device)
    return _default


class B200_lVector:
    """lVector<T> on the B200: a device buffer of `size` values."""

    def __init__(self, size: int, name: str = "", platform: Platform | None = None, dtype=np.float64,
                 _wrap_ptr: int | None = None, _keep=None):
        self.platform = platform or init_platform()
        self.name = name
        self.dtype = _dt(dtype)
        self.handle = C.c_void_p()
        self._keep = _keep
        if _wrap_ptr is None:
            call("b200la_vec_create", self.platform.handle, int(size), self.dtype, C.byref(self.handle))
        else:
            call("b200la_vec_wrap", self.platform.handle, int(size), self.dtype, C.c_void_p(_wrap_ptr),
                 C.byref(self.handle))
        self._size = int(size)

    # --- lVector API ---
    def get_size(self) -> int:
        return self._size

    def Zeros(self):
        call("b200la_vec_zeros", self.handle)

    def SetBlockValues(self, start: int, end: int, values):
        if start != 0 or end != self._size:
            raise B200LAError(-1, "SetBlockValues: only the full range is supported")
        a = np.ascontiguousarray(values, _NP[self.dtype])
        call("b200la_vec_upload", self.handle, a.ctypes.data_as(C.c_void_p), a.shape[0])

    def GetBlockValues(self, start: int = 0, end: int | None = None) -> np.ndarray:
        end = self._size if end is None else end
        out = np.empty(self._size, _NP[self.dtype])
        call("b200la_vec_download", self.handle, out.ctypes.data_as(C.c_void_p), self._size)
        return out[start:end]

    def SetValues(self, index, values):
        idx = np.ascontiguousarray(index, np.int32)
        v = np.ascontiguousarray(values, _NP[self.dtype])
        call("b200la_vec_set_values", self.handle, idx.ctypes.data_as(C.c_void_p),
             v.ctypes.data_as(C.c_void_p), idx.shape[0])

    def GetValues(self, index) -> np.ndarray:
        idx = np.ascontiguousarray(index, np.int32)
        out = np.empty(idx.shape[0], _NP[self.dtype])
        call("b200la_vec_get_values", self.handle, idx.ctypes.data_as(C.c_void_p),
             out.ctypes.data_as(C.c_void_p), idx.shape[0])
        return out

    def CopyFrom(self, other: "B200_lVector"):
        call("b200la_vec_copy", self.handle, other.handle)

    def CastFrom(self, other: "B200_lVector"):
        call("b200la_vec_cast", self.handle, other.handle)

    def CloneWithoutContent(self) -> "B200_lVector":
        return B200_lVector(self._size, self.name, self.platform, self.dtype)

    def Dot(self, other: "B200_lVector") -> float:
        out = C.c_double()
        call("b200la_vec_dot", self.handle, other.handle, C.byref(out))
        return out.value

    def Norm2(self) -> float:
        out = C.c_double()
        call("b200la_vec_norm2", self.handle, C.byref(out))
        return out.value

    def Axpy(self, vec: "B200_lVector", scalar: float):
        """this += scalar * vec"""
        call("b200la_vec_axpy", self.handle, vec.handle, float(scalar))

    def ScaleAdd(self, scalar: float, vec: "B200_lVector"):
        """this = scalar * this + vec"""
        call("b200la_vec_scaleadd", self.handle, float(scalar), vec.handle)

    def Scale(self, scalar: float):
        call("b200la_vec_scale", self.handle, float(scalar))

    def ElementWiseMult(self, vec: "B200_lVector"):
        call("b200la_vec_elementwise_mult", self.handle, vec.handle)

    def GetBuffer(self) -> int:
        p = C.c_void_p()
        call("b200la_vec_info", self.handle, None, None, C.byref(p))
        return p.value or 0

    def Clear(self):
        if self.handle:
            load().b200la_vec_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self, _fin=_finalizing):  # bound at definition: globals are gone at exit
        if _fin():
            return
        try:
            self.Clear()
        except Exception:
            pass

    # --- interop ---
    @classmethod
    def from_numpy(cls, a, name: str = "", platform: Platform | None = None, dtype=None):
        a = np.asarray(a)
        v = cls(a.shape[0], name, platform, dtype if dtype is not None else a.dtype)
        v.SetBlockValues(0, a.shape[0], a)
        return v

    @classmethod
    def from_torch(cls, t, name: str = "", platform: Platform | None = None):
        """Non-owning view of a contiguous 1-D CUDA tensor (kept alive)."""
        import torch
        assert t.is_cuda and t.dim() == 1 and t.is_contiguous()
        dt = {torch.float64: F64, torch.float32: F32}[t.dtype]
        return cls(t.shape[0], name, platform, dt, _wrap_ptr=t.data_ptr(), _keep=t)

    def numpy(self) -> np.ndarray:
        return self.GetBlockValues()


class B200_CSR_lMatrix:
    """CSR_lMatrix<T> on the B200 (int32 indices)."""

    def __init__(self, rowptr, col, val, num_col: int | None = None, name: str = "",
                 platform: Platform | None = None, dtype=np.float64):
        self.platform = platform or init_platform()
        self.name = name
        self.dtype = _dt(dtype)
        rp = np.ascontiguousarray(rowptr, np.int32)
        cl = np.ascontiguousarray(col, np.int32)
        vv = np.ascontiguousarray(val)
        if vv.dtype not in (np.float64, np.float32):
            vv = vv.astype(np.float64)
        nrow = rp.shape[0] - 1
        ncol = nrow if num_col is None else int(num_col)
        self.handle = C.c_void_p()
        call("b200la_csr_upload", self.platform.handle, nrow, ncol, cl.shape[0],
             rp.ctypes.data_as(C.c_void_p), cl.ctypes.data_as(C.c_void_p), vv.ctypes.data_as(C.c_void_p),
             _dt(vv.dtype), self.dtype, C.byref(self.handle))
        self._shape = (nrow, ncol, int(cl.shape[0]))

    @classmethod
    def TransformFromCOO(cls, rows, cols, data, num_rows: int, num_cols: int, name: str = "",
                         platform: Platform | None = None, dtype=np.float64) -> "B200_CSR_lMatrix":
        """CPU_CSR_lMatrix::TransformFromCOO (lmp/lmatrix_csr_cpu.cc:883-906) on
        the device: triplets in any order (host arrays, or torch CUDA tensors
        int32/int32/float, read in place), duplicates kept, the reference's CSR
        order bit for bit."""
        platform = platform or init_platform()
        dev = all(hasattr(a, "is_cuda") and a.is_cuda for a in (rows, cols, data))
        if dev:
            import torch
            assert rows.dtype == torch.int32 and cols.dtype == torch.int32
            nnz = int(rows.numel())
            vdt = F64 if data.dtype == torch.float64 else F32
            ptrs = [C.c_void_p(t.data_ptr()) for t in (rows, cols, data)]
        else:
            r = np.ascontiguousarray(rows, np.int32)
            c = np.ascontiguousarray(cols, np.int32)
            v = np.ascontiguousarray(data)
            if v.dtype not in (np.float64, np.float32):
                v = v.astype(np.float64)
            nnz = int(r.shape[0])
            vdt = _dt(v.dtype)
            keep = (r, c, v)
            ptrs = [a.ctypes.data_as(C.c_void_p) for a in keep]
        h = C.c_void_p()
        call("b200la_coo_upload", platform.handle, int(num_rows), int(num_cols), nnz, *ptrs, vdt, _dt(dtype),
             1 if dev else 0, C.byref(h))
        return cls._from_handle(h, platform, _dt(dtype), (int(num_rows), int(num_cols), nnz), name)

    def csr(self, out=None) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
        """The stored CSR arrays (rowptr, col, val) copied to host memory, into
        out = (rowptr, col, val) when given (contiguous arrays of at least
        nrow + 1, nnz and nnz elements of int32, int32 and the value type,
        e.g. views of pinned buffers)."""
        nrow, _, nnz = self._shape
        vdt = np.float64 if self.dtype == F64 else np.float32
        if out is None:
            rp = np.empty(nrow + 1, np.int32)
            cl = np.empty(max(nnz, 1), np.int32)
            vv = np.empty(max(nnz, 1), vdt)
        else:
            rp, cl, vv = out
            for a, need, dt in ((rp, nrow + 1, np.int32), (cl, nnz, np.int32), (vv, nnz, vdt)):
                if a.dtype != dt or not a.flags.c_contiguous or a.size < need:
                    raise B200LAError(-1, "csr: out arrays of the wrong type, layout or size")
        call("b200la_mat_download", self.handle, rp.ctypes.data_as(C.c_void_p), cl.ctypes.data_as(C.c_void_p),
             vv.ctypes.data_as(C.c_void_p))
        return rp[:nrow + 1], cl[:nnz], vv[:nnz]

    @classmethod
    def _from_handle(cls, handle, platform, dtype, shape, name=""):
        m = cls.__new__(cls)
        m.platform, m.name, m.dtype, m.handle, m._shape = platform, name, dtype, handle, shape
        return m

    def get_num_row(self) -> int:
        return self._shape[0]

    def get_num_col(self) -> int:
        return self._shape[1]

    def get_nnz(self) -> int:
        return self._shape[2]

    def VectorMult(self, invec: B200_lVector, outvec: B200_lVector):
        call("b200la_spmv", self.handle, invec.handle, outvec.handle)

    def VectorMultAdd(self, invec: B200_lVector, outvec: B200_lVector):
        call("b200la_spmv_add", self.handle, invec.handle, outvec.handle)

    def VectorMultNoDiag(self, invec: B200_lVector, outvec: B200_lVector):
        """outvec = (A - diag(A)) invec (CPU_CSR_lMatrix::VectorMultNoDiag)."""
        call("b200la_spmv_nodiag", self.handle, invec.handle, outvec.handle)

    def extract_invdiagelements(self, vec: B200_lVector):
        call("b200la_mat_inv_diag", self.handle, vec.handle)

    def ZeroRows(self, index_set, alpha: float = 1.0):
        idx = np.ascontiguousarray(index_set, np.int32)
        call("b200la_mat_zero_rows", self.handle, idx.ctypes.data_as(C.c_void_p), idx.shape[0], float(alpha))

    def CastTo(self, dtype) -> "B200_CSR_lMatrix":
        h = C.c_void_p()
        call("b200la_mat_cast", self.handle, _dt(dtype), C.byref(h))
        return B200_CSR_lMatrix._from_handle(h, self.platform, _dt(dtype), self._shape, self.name)

    def set_format(self, fmt: int, param: int):
        call("b200la_mat_set_format", self.handle, fmt, param)

    def set_sell(self, C: int = 32, sigma: int = 1, width: int = 1, col16: bool = False):
        """SELL-C-sigma schedule: slices of C (8/16/32) rows, rows sorted by
        length within windows of sigma rows, width entries per vector load,
        int16 column offsets with col16."""
        call("b200la_mat_to_sell", self.handle, int(C), int(sigma), int(width), 1 if col16 else 0)

    def get_sell(self) -> tuple[int, int]:
        """(C, sigma) of the current sliced schedule."""
        c, sg = C.c_int(), C.c_int()
        call("b200la_mat_get_sell", self.handle, C.byref(c), C.byref(sg), None)
        return c.value, sg.value

    def sell_padded(self) -> int:
        """Stored entries of the current sliced copy, padding included."""
        c, sg, pd = C.c_int(), C.c_int(), C.c_int64()
        call("b200la_mat_get_sell", self.handle, C.byref(c), C.byref(sg), C.byref(pd))
        return pd.value

    def get_format(self) -> tuple[int, int]:
        f, p = C.c_int(), C.c_int()
        call("b200la_mat_get_format", self.handle, C.byref(f), C.byref(p))
        return f.value, p.value

    def tune(self) -> tuple[int, int, float]:
        f, p, us = C.c_int(), C.c_int(), C.c_double()
        call("b200la_mat_tune", self.handle, C.byref(f), C.byref(p), C.byref(us))
        return f.value, p.value, us.value

    def Clear(self):
        if self.handle:
            load().b200la_mat_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self, _fin=_finalizing):  # bound at definition: globals are gone at exit
        if _fin():
            return
        try:
            self.Clear()
        except Exception:
            pass


def init_vector(size: int, name: str = "", platform: Platform | None = None, dtype=np.float64) -> B200_lVector:
    return B200_lVector(size, name, platform, dtype)


def init_matrix(rowptr, col, val, num_col=None, name: str = "", platform: Platform | None = None,
                dtype=np.float64) -> B200_CSR_lMatrix:
    return B200_CSR_lMatrix(rowptr, col, val, num_col, name, platform, dtype)


class IterateControl:
    """IterateControl(maxits, atol, rtol, dtol); defaults of
    common/iterate_control.cc:26-29."""

    def __init__(self, maxits: int = 1000, atol: float = 1e-12, rtol: float = 1e-8, dtol: float = 1e8):
        self.maxits, self.atol, self.rtol, self.dtol = int(maxits), float(atol), float(rtol), float(dtol)


class PreconditionerBlockJacobiStand:
    """Block-Jacobi over the local diagonal block with lmp's Jacobi inside."""

    def __init__(self):
        self.kind = None

    def Init_Jacobi(self):
        self.kind = "Jacobi"

    def SetupOperator(self, op):
        self.op = op


class CG:
    """CG<LAD>: the device PCG solver behind the reference's solver API."""

    def __init__(self):
        self.method = "NoPreconditioning"
        self.control = IterateControl()
        self.op = None
        self.precond = None
        self._solver = C.c_void_p()
        self._key = None
        self.iter_ = 0
        self.res_ = self.res_init_ = self.res_rel_ = 0.0
        self.state_ = 0

    def InitParameter(self, method: str):
        assert method in ("NoPreconditioning", "Preconditioning", "RightPreconditioning",
                          "LeftPreconditioning")
        self.method = method

    def InitControl(self, maxits: int, atol: float, rtol: float, dtol: float):
        self.control = IterateControl(maxits, atol, rtol, dtol)
        self._release()

    def SetupOperator(self, op: B200_CSR_lMatrix):
        self.op = op
        self._release()

    def SetupPreconditioner(self, precond: PreconditionerBlockJacobiStand):
        # LinearSolver::SetupPreconditioner switches CG to right preconditioning
        # (linear_solver.h:97-100)
        self.precond = precond
        self.method = "RightPreconditioning"
        self._release()

    def _release(self):
        if self._solver:
            load().b200la_cg_destroy(self._solver)
            self._solver = C.c_void_p()

    def _ensure(self):
        if self._solver:
            return
        if self.op is None:
            raise B200LAError(-1, "CG: SetupOperator was not called")
        use_pc = self.method != "NoPreconditioning"
        if use_pc and (self.precond is None or self.precond.kind != "Jacobi"):
            raise B200LAError(-7, "CG: only the Jacobi preconditioner runs on this path")
        c = self.control
        prm = CgParams(c.maxits, c.atol, c.rtol, c.dtol, 1 if use_pc else 0, 0)
        call("b200la_cg_create", self.op.handle, C.byref(prm), C.byref(self._solver))

    def Solve(self, b: B200_lVector, x: B200_lVector) -> int:
        self._ensure()
        r = CgResult()
        call("b200la_cg_solve", self._solver, b.handle, x.handle, C.byref(r))
        self.iter_, self.state_ = r.iters, r.state
        self.res_, self.res_init_, self.res_rel_ = r.res, r.res_init, r.res_rel
        return r.solver_state

    def iter(self) -> int:
        return self.iter_

    def res(self) -> float:
        return self.res_

    def res_init(self) -> float:
        return self.res_init_

    def res_rel(self) -> float:
        return self.res_rel_

    def __del__(self, _fin=_finalizing):  # bound at definition: globals are gone at exit
        if _fin():
            return
        try:
            self._release()
        except Exception:
            pass


def cg(x: B200_lVector, b: B200_lVector, matrix: B200_CSR_lMatrix, rel_eps: float, abs_eps: float, max_iter: int,
       print_level: int = -1, lPrecond=None) -> tuple[int, int]:
    """The lmp cg() (lmp/solvers/cg.cc:35-41, CGFunctor, lmp/solvers/cg.h:93-209)
    as one device solve: plain CG from x, stop after an iteration once
    ||r|| <= max(rel_eps ||r0||, abs_eps), at most max_iter iterations.
    Returns (0, index) where index is what cg() leaves in max_iter: the
    0-based index of the breaking iteration, or max_iter.  lPrecond is
    accepted and, as in the reference (which computes z but never uses it,
    cg.h:153 vs :157), has no effect on the iterates."""
    del print_level, lPrecond
    prm = CgParams(int(max_iter), float(abs_eps), float(rel_eps), 1e300, 0, 1)
    s = C.c_void_p()
    call("b200la_cg_create", matrix.handle, C.byref(prm), C.byref(s))
    try:
        r = CgResult()
        call("b200la_cg_solve", s, b.handle, x.handle, C.byref(r))
    finally:
        load().b200la_cg_destroy(s)
    return 0, r.iters


def setup_CG_solver(maxits: int = 1000, atol: float = 1e-12, rtol: float = 1e-10, dtol: float = 1e6,
                    use_precond: bool = True) -> CG:
    """setup_CG_solver defaults (linear_solver/cg.h:271-293)."""
    s = CG()
    s.InitControl(maxits, atol, rtol, dtol)
    if use_precond:
        p = PreconditionerBlockJacobiStand()
        p.Init_Jacobi()
        s.SetupPreconditioner(p)
    return s


class _DeviceSolver:
    """Common part of the solvers that run on b200la_solver (Jacobi, BiCGSTAB)."""

    _name = "solver"

    def __init__(self):
        self.control = IterateControl()
        self.op = None
        self._s = C.c_void_p()
        self.iter_ = 0
        self.res_ = self.res_init_ = self.res_rel_ = 0.0
        self.state_ = 0
        self.restarts_ = 0

    def InitControl(self, maxits: int, atol: float, rtol: float, dtol: float):
        self.control = IterateControl(maxits, atol, rtol, dtol)
        self._release()

    def SetRelativeTolerance(self, reltol: float):
        c = self.control
        self.InitControl(c.maxits, c.atol, reltol, c.dtol)

    def SetupOperator(self, op: B200_CSR_lMatrix):
        self.op = op
        self._release()

    def _params(self) -> "_lib.SolverParams":
        raise NotImplementedError

    def _release(self):
        if self._s:
            load().b200la_solver_destroy(self._s)
            self._s = C.c_void_p()

    def _ensure(self):
        if self._s:
            return
        if self.op is None:
            raise B200LAError(-1, f"{self._name}: SetupOperator was not called")
        prm = self._params()
        call("b200la_solver_create", self.op.handle, C.byref(prm), C.byref(self._s))

    def _solve(self, b: B200_lVector, x: B200_lVector) -> "_lib.SolverResult":
        self._ensure()
        r = _lib.SolverResult()
        call("b200la_solver_solve", self._s, b.handle, x.handle, C.byref(r))
        self.state_, self.restarts_ = r.state, r.restarts
        self.res_, self.res_init_, self.res_rel_ = r.res, r.res_init, r.res_rel
        return r

    def profile(self, b: B200_lVector, x: B200_lVector, passes: int = 20) -> list[float]:
        """Mean milliseconds per launch of each kernel of one pass."""
        self._ensure()
        ms = (C.c_double * 5)()
        call("b200la_solver_profile", self._s, b.handle, x.handle, int(passes), ms)
        return list(ms)

    def iter(self) -> int:
        return self.iter_

    def res(self) -> float:
        return self.res_

    def res_init(self) -> float:
        return self.res_init_

    def res_rel(self) -> float:
        return self.res_rel_

    def __del__(self, _fin=_finalizing):  # bound at definition: globals are gone at exit
        if _fin():
            return
        try:
            self._release()
        except Exception:
            pass


class Jacobi(_DeviceSolver):
    """Jacobi<LAD> (linear_solver/jacobi.h:30-80, jacobi.cc): the stationary
    Jacobi solver and smoother.  SetSolveMode(0 SolveNormal, 1 SolveDamped,
    2 SmoothNormal, 3 SmoothDamped), SetNumIter (smoothing sweeps),
    SetInnerIter (sweeps between residual tests), SetDampingParameter(w).
    As in the reference, the smoothing modes add their sweeps to iter() and
    the solve modes restart it from 0.  Prepare(op, sample) is SetupOperator;
    the asynchronous ghost flag has no meaning on one device and is stored
    only."""

    _name = "Jacobi"

    def __init__(self):
        super().__init__()
        self.solve_mode, self.smooth_iter, self.inner_iter, self.w, self.async_ = 0, 1, 1, 1.0, False

    def Prepare(self, op: B200_CSR_lMatrix, sample: B200_lVector | None = None):
        self.SetupOperator(op)

    def SetSolveMode(self, mode: int):
        if not 0 <= int(mode) <= 3:
            raise B200LAError(-1, f"Jacobi: unknown solve mode {mode}")
        self.solve_mode = int(mode)
        self._release()

    def SetNumIter(self, it: int):
        if int(it) <= 0:
            raise B200LAError(-1, "Jacobi: SetNumIter needs a positive count")
        self.smooth_iter = int(it)
        self._release()

    def SetInnerIter(self, it: int):
        if int(it) <= 0:
            raise B200LAError(-1, "Jacobi: SetInnerIter needs a positive count")
        self.inner_iter = int(it)
        self._release()

    def SetDampingParameter(self, w: float):
        if not float(w) > 0.0:
            raise B200LAError(-1, "Jacobi: the damping parameter must be positive")
        self.w = float(w)
        self._release()

    def SetAsyncFlag(self, flag: bool):
        self.async_ = bool(flag)

    def _params(self):
        c = self.control
        return _lib.SolverParams(_lib.METHOD_JACOBI, c.maxits, c.atol, c.rtol, c.dtol, 1, self.solve_mode,
                                 self.inner_iter, self.smooth_iter, self.w, 0)

    def Solve(self, b: B200_lVector, x: B200_lVector) -> int:
        r = self._solve(b, x)
        if self.solve_mode >= 2:
            self.iter_ += r.iters
        else:
            self.iter_ = r.iters
        return r.solver_state


class BiCGSTAB(_DeviceSolver):
    """BiCGSTAB<LAD> (linear_solver/bicgstab.h:37-473):
    InitParameter("NoPreconditioning" | "RightPreconditioning" |
    "LeftPreconditioning"), SetupPreconditioner (switches to right
    preconditioning, linear_solver.h:97-100), Solve.  Left preconditioning
    returns kSolverError as in the reference (bicgstab.h:485-495).  iter()
    reports the iterations taken (the reference never stores its local
    count in iter_); restarts() the restarts."""

    _name = "BiCGSTAB"

    def __init__(self):
        super().__init__()
        self.method = "NoPreconditioning"
        self.precond = None

    def InitParameter(self, method: str):
        if method not in ("NoPreconditioning", "RightPreconditioning", "LeftPreconditioning"):
            raise B200LAError(-1, f"BiCGSTAB: unknown method {method!r}")
        self.method = method
        self._release()

    def SetupPreconditioner(self, precond: PreconditionerBlockJacobiStand):
        self.precond = precond
        self.method = "RightPreconditioning"
        self._release()

    def _params(self):
        use_pc = self.method == "RightPreconditioning"
        if use_pc and (self.precond is None or self.precond.kind != "Jacobi"):
            raise B200LAError(-7, "BiCGSTAB: only the Jacobi preconditioner runs on this path")
        c = self.control
        return _lib.SolverParams(_lib.METHOD_BICGSTAB, c.maxits, c.atol, c.rtol, c.dtol, 1 if use_pc else 0,
                                 0, 1, 1, 1.0, 0)

    def Solve(self, b: B200_lVector, x: B200_lVector) -> int:
        if self.method == "LeftPreconditioning":
            return kSolverError
        r = self._solve(b, x)
        self.iter_ = r.iters
        return r.solver_state

    def restarts(self) -> int:
        return self.restarts_


class GMRES(_DeviceSolver):
    """GMRES<LAD, PreLAD> (linear_solver/gmres.h:46-746): InitParameter(size_basis,
    "NoPreconditioning" | "RightPreconditioning" | "LeftPreconditioning"),
    SetupPreconditioner (switches to right preconditioning), InitControl,
    Solve.  Restarted after size_basis steps (default 100, gmres.h:145), modified
    Gram-Schmidt; left preconditioning with a preconditioner set returns
    kSolverError as in the reference (gmres.h:394-404), and without one the
    solve is unpreconditioned (gmres.h:213-219)."""

    _name = "GMRES"

    def __init__(self):
        super().__init__()
        self.size_basis_ = 100
        self.method = "NoPreconditioning"
        self.precond = None

    def InitParameter(self, size_basis: int, method: str):
        if method not in ("NoPreconditioning", "RightPreconditioning", "LeftPreconditioning"):
            raise B200LAError(-1, f"GMRES: unknown method {method!r}")
        self.size_basis_, self.method = int(size_basis), method
        self._release()

    def size_basis(self) -> int:
        return self.size_basis_

    def SetupPreconditioner(self, precond: PreconditionerBlockJacobiStand):
        self.precond = precond
        self.method = "RightPreconditioning"
        self._release()

    def _params(self):
        # SolveImpl (gmres.h:194-221): right preconditioning only with a
        # preconditioner set, otherwise SolveNoPrecond
        use_pc = self.method == "RightPreconditioning" and self.precond is not None
        if use_pc and self.precond.kind != "Jacobi":
            raise B200LAError(-7, "GMRES: only the Jacobi preconditioner runs on this path")
        c = self.control
        return _lib.SolverParams(_lib.METHOD_GMRES, c.maxits, c.atol, c.rtol, c.dtol, 1 if use_pc else 0,
                                 0, 1, 1, 1.0, self.size_basis_)

    def Solve(self, b: B200_lVector, x: B200_lVector) -> int:
        if self.size_basis_ <= 0 or (self.method == "LeftPreconditioning" and self.precond is not None):
            return kSolverError
        r = self._solve(b, x)
        self.iter_ = r.iters
        return r.solver_state


class MPIR:
    """MPIR<LADescriptorCoupledD, LADescriptorCoupledS> (linear_solver/mpir.h:29-150,
    mpir.cc:52-250) with B200 operands.

    Generic form, as in the reference: SetHighPrecMatrix / SetLowPrecMatrix
    (or SetupOperator(A64), which makes the FP32 copy), the work vectors
    (made on first use if not set), SetLowPrecErrCorSolver /
    SetHighPrecErrCorSolver and the four smoothers (any of CG, Jacobi,
    BiCGSTAB, GMRES here, each running on the device), their
    Set*Parameters, Use*Smoother and SetMpirParameters(max_ech, max_ecl,
    abs_tol, rel_tol, div_tol); Solve runs SolveImpl's loop: FP64 residual,
    then while ContinueIteration(): high pre-smoothing, a low-precision
    error-correction pass (cast, low pre-smoothing, correction solve, low
    post-smoothing, cast back) while max_ecl allows, else a high-precision
    one, x += correction, high post-smoothing, FP64 residual, res0 = res.
    Kept from the reference: res0_ moves to the latest residual after every
    pass (mpir.cc:240), the component parameters default to 0 iterations,
    and the pass counters n_ech_, n_ecl_ are not reset by Solve.

    Fast form (no error-correction solver set): one fused device solve
    (b200la_mp) with an FP32 Jacobi-PCG as the low-precision solver, outer
    test relative to the initial residual, SetLowPrecErrCorSolverParameters
    applying to that PCG; max_ech must be 0 there."""

    def __init__(self):
        self.op = None
        self.max_ech, self.max_ecl, self.abs_tol, self.rel_tol, self.div_tol = 0, 50, 0.0, 1e-10, 1e6
        self.inner_maxits, self.inner_rtol = 100000, 1e-5
        self.precond = True
        self.tune = True
        # fast form: 0 = FP32 inner PCG; 1 = FP32 matrix values under FP64 vectors and dots
        self.inner_storage = 0
        # fast form: False = each pass continues the inner PCG from the FP64 residual with
        # its search direction kept; True = restart it each pass (as MPIR restarts its solver)
        self.restart_inner = False
        self._s = C.c_void_p()
        self.iter_ = 0
        self.outer_ = 0
        self.res_ = self.res_init_ = self.res_rel_ = 0.0
        # generic form
        self.Ah = self.Al = None
        self.resh = self.corh = self.resl = self.corl = None
        self.solvers = {}                 # role -> solver; roles: ech, ecl, preh, posth, prel, postl
        self.params = {r: (0, 0.0, 0.0, 0.0) for r in ("ech", "ecl", "preh", "posth", "prel", "postl")}
        self.use = {"preh": False, "posth": False, "prel": False, "postl": False}
        self.n_ech = self.n_ecl = 0
        self.accu = {r: 0 for r in self.params}
        self.res0_ = 0.0

    # ---- operators and work vectors
    def SetupOperator(self, op: B200_CSR_lMatrix):
        self.op = op
        self.Ah = op
        self._release()

    def SetInnerRestart(self, restart: bool):
        """Fast form: restart the inner PCG from p = z at every refinement
        pass (True, as MPIR restarts its error-correction solver) or keep its
        search direction across passes (False, the default)."""
        self.restart_inner = bool(restart)
        self._release()

    def SetInnerStorage(self, f64_vectors: bool):
        """Fast form: keep the FP32 matrix values but run the inner PCG's
        vectors, dot products and Jacobi scaling in FP64 (True), or all in
        FP32 (False, the default)."""
        self.inner_storage = 1 if f64_vectors else 0
        self._release()

    def SetHighPrecMatrix(self, mh: B200_CSR_lMatrix):
        self.SetupOperator(mh)

    def SetLowPrecMatrix(self, ml: B200_CSR_lMatrix):
        self.Al = ml

    def SetHighPrecResVector(self, v: B200_lVector):
        self.resh = v

    def SetHighPrecCorVector(self, v: B200_lVector):
        self.corh = v

    def SetLowPrecResVector(self, v: B200_lVector):
        self.resl = v

    def SetLowPrecCorVector(self, v: B200_lVector):
        self.corl = v

    def SetupPreconditioner(self, precond):
        pass  # MPIR::SetupPreconditioner does nothing (mpir.cc:47-50)

    # ---- components
    def SetHighPrecPreSmoother(self, s):
        self.solvers["preh"] = s

    def SetHighPrecPostSmoother(self, s):
        self.solvers["posth"] = s

    def SetLowPrecPreSmoother(self, s):
        self.solvers["prel"] = s

    def SetLowPrecPostSmoother(self, s):
        self.solvers["postl"] = s

    def SetHighPrecErrCorSolver(self, s):
        self.solvers["ech"] = s

    def SetLowPrecErrCorSolver(self, s):
        self.solvers["ecl"] = s

    def UseHighPrecPreSmoother(self, use: bool):
        self.use["preh"] = bool(use)

    def UseHighPrecPostSmoother(self, use: bool):
        self.use["posth"] = bool(use)

    def UseLowPrecPreSmoother(self, use: bool):
        self.use["prel"] = bool(use)

    def UseLowPrecPostSmoother(self, use: bool):
        self.use["postl"] = bool(use)

    def SetMpirParameters(self, max_ech: int, max_ecl: int, abs_tol: float, rel_tol: float, div_tol: float):
        self.max_ech, self.max_ecl = int(max_ech), int(max_ecl)
        self.abs_tol, self.rel_tol, self.div_tol = float(abs_tol), float(rel_tol), float(div_tol)
        self._release()

    def _set_params(self, role, max_iter, abs_tol, rel_tol, div_tol):
        self.params[role] = (int(max_iter), float(abs_tol), float(rel_tol), float(div_tol))
        self._reset(role)

    def _reset(self, role):
        sv = self.solvers.get(role)
        if sv is not None:
            sv.InitControl(*self.params[role])

    def SetHighPrecPreSmootherParameters(self, max_iter, abs_tol, rel_tol, div_tol):
        self._set_params("preh", max_iter, abs_tol, rel_tol, div_tol)

    def SetHighPrecPostSmootherParameters(self, max_iter, abs_tol, rel_tol, div_tol):
        self._set_params("posth", max_iter, abs_tol, rel_tol, div_tol)

    def SetLowPrecPreSmootherParameters(self, max_iter, abs_tol, rel_tol, div_tol):
        self._set_params("prel", max_iter, abs_tol, rel_tol, div_tol)

    def SetLowPrecPostSmootherParameters(self, max_iter, abs_tol, rel_tol, div_tol):
        self._set_params("postl", max_iter, abs_tol, rel_tol, div_tol)

    def SetHighPrecErrCorSolverParameters(self, max_iter, abs_tol, rel_tol, div_tol):
        self._set_params("ech", max_iter, abs_tol, rel_tol, div_tol)

    def SetLowPrecErrCorSolverParameters(self, max_iter: int, abs_tol: float, rel_tol: float, div_tol: float):
        self._set_params("ecl", max_iter, abs_tol, rel_tol, div_tol)
        self.inner_maxits, self.inner_rtol = int(max_iter), float(rel_tol)
        self._release()

    # ---- fast form
    def _release(self):
        if self._s:
            load().b200la_mp_destroy(self._s)
            self._s = C.c_void_p()

    def _ensure(self):
        if self._s:
            return
        if self.op is None:
            raise B200LAError(-1, "MPIR: SetupOperator was not called")
        if self.max_ech != 0:
            raise B200LAError(-7, "MPIR: high-precision correction passes need SetHighPrecErrCorSolver")
        prm = _lib.MpParams(self.max_ecl, self.abs_tol, self.rel_tol, self.div_tol, self.inner_maxits,
                            self.inner_rtol, 1 if self.precond else 0, 1 if self.tune else 0,
                            int(self.inner_storage), 1 if self.restart_inner else 0)
        call("b200la_mp_create", self.op.handle, C.byref(prm), C.byref(self._s))

    # ---- generic form: SolveImpl (mpir.cc:52-285), ContinueIteration (:288-297)
    def _continue(self) -> bool:
        r, r0 = self.res_, self.res0_
        return (r > self.abs_tol and r > r0 * self.rel_tol and r < self.div_tol and
                ((self.n_ech < self.max_ech and r > self.params["ech"][1] and r > r0 * self.params["ech"][2]
                  and r < self.params["ech"][3]) or
                 (self.n_ecl < self.max_ecl and r > self.params["ecl"][1] and r > r0 * self.params["ecl"][2]
                  and r < self.params["ecl"][3])))

    def _residual(self, b, x):
        self.Ah.VectorMult(x, self.resh)
        self.resh.ScaleAdd(-1.0, b)        # coupled resh.ScaleAdd(b, -1)
        self.res_ = self.resh.Norm2()

    def _run(self, role, b, x):
        sv = self.solvers[role]
        sv.Solve(b, x)
        self.accu[role] += sv.iter()
        self.iter_ += sv.iter()

    def _solve_generic(self, b: B200_lVector, x: B200_lVector) -> int:
        if self.Ah is None:
            raise B200LAError(-1, "MPIR: SetupOperator was not called")
        n = self.Ah.get_num_row()
        plat = self.Ah.platform
        if self.Al is None:
            self.Al = self.Ah.CastTo(np.float32)
        for name, dt in (("resh", np.float64), ("corh", np.float64), ("resl", np.float32), ("corl", np.float32)):
            if getattr(self, name) is None:
                setattr(self, name, B200_lVector(n, name, platform=plat, dtype=dt))
        self.iter_ = 0
        self.accu = {r: 0 for r in self.params}
        for role, mat in (("preh", self.Ah), ("prel", self.Al), ("ecl", self.Al), ("postl", self.Al),
                          ("ech", self.Ah), ("posth", self.Ah)):
            if role in self.solvers and (role in ("ecl", "ech") or self.use.get(role)):
                self._reset(role)
                self.solvers[role].SetupOperator(mat)
            elif self.use.get(role):
                raise B200LAError(-1, f"MPIR: smoother {role} is used but not set")
        self._residual(b, x)
        self.res_init_ = self.res_
        self.res0_ = self.res_
        passes = 0
        while self._continue():
            passes += 1
            if self.use["preh"]:
                self._run("preh", b, x)
                self._residual(b, x)
            r, r0 = self.res_, self.res0_
            pe = self.params["ecl"]
            ph = self.params["ech"]
            if "ecl" in self.solvers and self.n_ecl < self.max_ecl and r > pe[1] and r > r0 * pe[2] and r < pe[3]:
                self.n_ecl += 1
                self.resl.CastFrom(self.resh)
                self.corl.Zeros()
                if self.use["prel"]:
                    self._run("prel", self.resl, self.corl)
                self._run("ecl", self.resl, self.corl)
                if self.use["postl"]:
                    self._run("postl", self.resl, self.corl)
                self.corh.CastFrom(self.corl)
            elif "ech" in self.solvers and self.n_ech < self.max_ech and r > ph[1] and r > r0 * ph[2] and r < ph[3]:
                self.n_ech += 1
                self.corh.Zeros()
                self._run("ech", self.resh, self.corh)
            x.Axpy(self.corh, 1.0)
            if self.use["posth"]:
                self._run("posth", b, x)
            self._residual(b, x)
            self.res0_ = self.res_
        self.outer_ = passes
        self.res_rel_ = self.res_ / self.res_init_ if self.res_init_ > 0 else 0.0
        if self.res_ < self.abs_tol or self.res_ < self.res0_ * self.rel_tol:
            return kSolverSuccess
        return kSolverExceeded

    def Solve(self, b: B200_lVector, x: B200_lVector) -> int:
        if "ecl" in self.solvers or "ech" in self.solvers:
            return self._solve_generic(b, x)
        self._ensure()
        r = _lib.MpResult()
        call("b200la_mp_solve", self._s, b.handle, x.handle, C.byref(r))
        self.iter_, self.outer_ = r.inner_iters, r.outer
        self.res_, self.res_init_, self.res_rel_ = r.res, r.res_init, r.res_rel
        self.state_ = r.state
        return r.solver_state

    def iter(self) -> int:
        return self.iter_

    def res(self) -> float:
        return self.res_

    def __del__(self, _fin=_finalizing):  # bound at definition: globals are gone at exit
        if _fin():
            return
        try:
            self._release()
        except Exception:
            pass
