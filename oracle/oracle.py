"""ctypes bindings of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

See pcg_oracle.c (restatement) and ref/ref_driver.cc (reference sources).
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_REF_PATH = os.path.join(_HERE, "_ref", "libhiflow_lmp_ref.so")

CTRL_ITERATE, CTRL_SUCCESS_ABS, CTRL_SUCCESS_REL, CTRL_FAIL_DIV, CTRL_FAIL_MAXITS = range(5)
IMPL_NAIVE, IMPL_OPENMP = 0, 1

_lib = None
_ref = None

_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_ip = C.POINTER(C.c_int)
_dp = C.POINTER(C.c_double)


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            raise RuntimeError(f"oracle not built: {_LIB_PATH} (run `make -C oracle`)")
        lib = C.CDLL(_LIB_PATH)
        for s, fp in (("d", _f64p), ("f", _f32p)):
            T = C.c_double if s == "d" else C.c_float
            getattr(lib, f"orc_spmv_{s}").argtypes = [C.c_int, _i32p, _i32p, fp, fp, fp]
            getattr(lib, f"orc_dot_{s}").argtypes = [C.c_int, fp, fp]
            getattr(lib, f"orc_dot_{s}").restype = T
            getattr(lib, f"orc_invdiag_{s}").argtypes = [C.c_int, _i32p, _i32p, fp, fp]
            getattr(lib, f"orc_cg_{s}").argtypes = [
                C.c_int, _i32p, _i32p, fp, fp, fp, C.c_int, C.c_double, C.c_double,
                C.c_double, C.c_int, fp, fp, _ip, _dp, _dp]
            getattr(lib, f"orc_lmp_cg_{s}").argtypes = [
                C.c_int, _i32p, _i32p, fp, fp, fp, T, T, _ip, fp]
            getattr(lib, f"orc_spmv_nodiag_{s}").argtypes = [C.c_int, _i32p, _i32p, fp, fp, fp]
            getattr(lib, f"orc_jacobi_{s}").argtypes = [
                C.c_int, _i32p, _i32p, fp, fp, fp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double,
                C.c_double, C.c_double, C.c_double, _ip, _dp, _dp]
            getattr(lib, f"orc_bicgstab_{s}").argtypes = [
                C.c_int, _i32p, _i32p, fp, fp, fp, C.c_int, fp, C.c_int, C.c_double, C.c_double,
                C.c_double, _ip, _ip, _dp, _dp]
            getattr(lib, f"orc_gmres_{s}").argtypes = [
                C.c_int, _i32p, _i32p, fp, fp, fp, C.c_int, fp, C.c_int, C.c_int, C.c_double,
                C.c_double, C.c_double, _ip, _dp, _dp]
        lib.orc_coo2csr_d.argtypes = [C.c_int, C.c_int, C.c_int, _i32p, _i32p, _f64p, _i32p, _i32p, _f64p, _i32p]
        lib.orc_iterate_check.argtypes = [C.c_int, C.c_double, C.c_int, C.c_double, C.c_double,
                                          C.c_double, _dp]
        lib.orc_mpir_d.argtypes = [C.c_int, _i32p, _i32p, _f64p, _f32p, _f64p, _f64p, C.c_int,
                                   C.c_double, C.c_double, C.c_double, C.c_int, _f64p, _f32p, _f64p, _f32p,
                                   _ip, _ip, _dp, _dp]
        lib.orc_mpcg_kept_d.argtypes = [C.c_int, _i32p, _i32p, _f64p, _f32p, _f64p, _f64p, C.c_int,
                                        C.c_double, C.c_double, C.c_double, C.c_int, _f32p, _f64p, _f32p,
                                        _ip, _ip, _dp, _dp]
        _lib = lib
    return _lib


def ref_available() -> bool:
    return os.path.exists(_REF_PATH)


def _load_ref():
    global _ref
    if _ref is None:
        if not ref_available():
            raise RuntimeError(f"reference checker not built: {_REF_PATH} (run `make -C oracle`)")
        lib = C.CDLL(_REF_PATH)
        for s, fp in (("d", _f64p), ("f", _f32p)):
            getattr(lib, f"ref_spmv_{s}").argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, _i32p, _i32p,
                                                     fp, fp, fp]
            getattr(lib, f"ref_cg_solve_{s}").argtypes = [
                C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _i32p, _i32p, fp, fp, fp, C.c_int,
                C.c_double, C.c_double, C.c_double, _ip, _dp, _dp, _dp]
        lib.ref_jacobi_solve_d.argtypes = [
            C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _i32p, _i32p, _f64p, _f64p, _f64p, C.c_int,
            C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, _ip, _dp, _dp, _dp]
        lib.ref_bicgstab_solve_d.argtypes = [
            C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _i32p, _i32p, _f64p, _f64p, _f64p, C.c_int,
            C.c_double, C.c_double, C.c_double, _ip, _ip, _dp, _dp, _dp]
        lib.ref_gmres_solve_d.argtypes = [
            C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _i32p, _i32p, _f64p, _f64p, _f64p, C.c_int,
            C.c_int, C.c_double, C.c_double, C.c_double, _ip, _dp, _dp, _dp]
        lib.ref_coo_to_csr_d.argtypes = [C.c_int, C.c_int, C.c_int, _i32p, _i32p, _f64p, _i32p, _i32p, _f64p]
        lib.ref_lmp_cg_d.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, _i32p, _i32p, _f64p, _f64p,
                                     _f64p, C.c_double, C.c_double, _ip]
        _ref = lib
    return _ref


def _sfx(dtype) -> tuple[str, type]:
    dt = np.dtype(dtype)
    if dt == np.float64:
        return "d", np.float64
    if dt == np.float32:
        return "f", np.float32
    raise TypeError(f"unsupported dtype {dt}")


def _csr(rowptr, col, val, dtype):
    return (np.ascontiguousarray(rowptr, np.int32), np.ascontiguousarray(col, np.int32),
            np.ascontiguousarray(val, dtype))


@dataclass
class OracleResult:
    x: np.ndarray
    iters: int
    res: float
    res_init: float
    state: int
    seconds: float = 0.0   # reference runs: time of the iteration loop alone

    @property
    def res_rel(self) -> float:
        return self.res / self.res_init if self.res_init > 0 else 0.0


def iterate_check(step: int, value: float, maxits: int, atol: float, rtol: float, dtol: float,
                  first: float) -> tuple[int, float]:
    f = C.c_double(first)
    st = _load().orc_iterate_check(step, value, maxits, atol, rtol, dtol, C.byref(f))
    return st, f.value


def spmv(rowptr, col, val, x, dtype=np.float64) -> np.ndarray:
    s, T = _sfx(dtype)
    rp, c, v = _csr(rowptr, col, val, T)
    n = rp.shape[0] - 1
    y = np.empty(n, T)
    getattr(_load(), f"orc_spmv_{s}")(n, rp, c, v, np.ascontiguousarray(x, T), y)
    return y


def dot(a, b, dtype=np.float64) -> float:
    s, T = _sfx(dtype)
    a = np.ascontiguousarray(a, T)
    return float(getattr(_load(), f"orc_dot_{s}")(a.shape[0], a, np.ascontiguousarray(b, T)))


def invdiag(rowptr, col, val, dtype=np.float64) -> np.ndarray:
    s, T = _sfx(dtype)
    rp, c, v = _csr(rowptr, col, val, T)
    n = rp.shape[0] - 1
    out = np.empty(n, T)
    bad = getattr(_load(), f"orc_invdiag_{s}")(n, rp, c, v, out)
    if bad >= 0:
        raise ValueError(f"row {bad} has no nonzero diagonal")
    return out


def cg(rowptr, col, val, b, x0=None, *, maxits=1000, atol=1e-12, rtol=1e-8, dtol=1e8,
       precond=True, dtype=np.float64) -> OracleResult:
    """CG<LAD>::SolvePrecond (precond) / SolveNoPrecond restated in C."""
    s, T = _sfx(dtype)
    rp, c, v = _csr(rowptr, col, val, T)
    n = rp.shape[0] - 1
    x = np.zeros(n, T) if x0 is None else np.array(x0, T)
    inv = invdiag(rp, c, v, T) if precond else np.zeros(1, T)
    work = np.empty(5 * n, T)
    it, res, res0 = C.c_int(), C.c_double(), C.c_double()
    st = getattr(_load(), f"orc_cg_{s}")(n, rp, c, v, np.ascontiguousarray(b, T), x, int(maxits),
                                         atol, rtol, dtol, int(bool(precond)), inv, work,
                                         C.byref(it), C.byref(res), C.byref(res0))
    return OracleResult(x, it.value, res.value, res0.value, st)


def lmp_cg(rowptr, col, val, b, x0=None, *, rel_eps=1e-10, abs_eps=0.0, max_iter=10000,
           dtype=np.float64) -> OracleResult:
    """lmp cg() restated in C; iters is cg()'s returned max_iter."""
    s, T = _sfx(dtype)
    rp, c, v = _csr(rowptr, col, val, T)
    n = rp.shape[0] - 1
    x = np.zeros(n, T) if x0 is None else np.array(x0, T)
    mi = C.c_int(int(max_iter))
    getattr(_load(), f"orc_lmp_cg_{s}")(n, rp, c, v, np.ascontiguousarray(b, T), x, rel_eps,
                                        abs_eps, C.byref(mi), np.empty(3 * n, T))
    return OracleResult(x, mi.value, float("nan"), float("nan"), 0)


def mpir(rowptr, col, val, b, *, rtol=1e-10, inner_rtol=1e-4, inner_maxits=100000,
         max_outer=50, floor=0.0) -> tuple[OracleResult, int]:
    """FP64 refinement around a float Jacobi-PCG (MPIR structure)."""
    rp, c, v = _csr(rowptr, col, val, np.float64)
    v32 = v.astype(np.float32)
    n = rp.shape[0] - 1
    x = np.zeros(n, np.float64)
    inv = invdiag(rp, c, v, np.float64)
    inv32 = invdiag(rp, c, v32, np.float32)
    outer, inner, res, res0 = C.c_int(), C.c_int(), C.c_double(), C.c_double()
    st = _load().orc_mpir_d(n, rp, c, v, v32, np.ascontiguousarray(b, np.float64), x, max_outer,
                            rtol, inner_rtol, floor, inner_maxits, inv, inv32, np.empty(3 * n),
                            np.empty(8 * n, np.float32), C.byref(outer), C.byref(inner),
                            C.byref(res), C.byref(res0))
    return OracleResult(x, inner.value, res.value, res0.value, st), outer.value


def mpcg_kept(rowptr, col, val, b, *, rtol=1e-10, inner_rtol=0.1, inner_maxits=100000,
              max_outer=50, floor=0.0) -> tuple[OracleResult, int]:
    """Mixed-precision Jacobi-PCG with residual replacement (the device's
    default fused refinement: float inner PCG whose recurrence residual is
    replaced by the double b - A x every inner_rtol reduction, search
    direction kept).  Returns (result with the total inner iterations,
    passes)."""
    rp, c, v = _csr(rowptr, col, val, np.float64)
    v32 = v.astype(np.float32)
    n = rp.shape[0] - 1
    x = np.zeros(n, np.float64)
    inv32 = invdiag(rp, c, v32, np.float32)
    outer, inner, res, res0 = C.c_int(), C.c_int(), C.c_double(), C.c_double()
    st = _load().orc_mpcg_kept_d(n, rp, c, v, v32, np.ascontiguousarray(b, np.float64), x, max_outer,
                                 rtol, inner_rtol, floor, inner_maxits, inv32, np.empty(n),
                                 np.empty(6 * n, np.float32),
                                 C.byref(outer), C.byref(inner), C.byref(res), C.byref(res0))
    return OracleResult(x, inner.value, res.value, res0.value, st), outer.value


def spmv_nodiag(rowptr, col, val, x, dtype=np.float64) -> np.ndarray:
    """CPU_CSR_lMatrix::VectorMultNoDiag restated in C."""
    s, T = _sfx(dtype)
    rp, c, v = _csr(rowptr, col, val, T)
    n = rp.shape[0] - 1
    y = np.empty(n, T)
    getattr(_load(), f"orc_spmv_nodiag_{s}")(n, rp, c, v, np.ascontiguousarray(x, T), y)
    return y


# Jacobi<LAD>::SetSolveMode values (linear_solver/jacobi.cc SolveImpl)
JACOBI_SOLVE_NORMAL, JACOBI_SOLVE_DAMPED, JACOBI_SMOOTH_NORMAL, JACOBI_SMOOTH_DAMPED = range(4)


def jacobi(rowptr, col, val, b, x0=None, *, mode=JACOBI_SOLVE_NORMAL, maxits=1000, inner_iter=1,
           smooth_iter=1, w=1.0, atol=1e-12, rtol=1e-8, dtol=1e8, dtype=np.float64) -> OracleResult:
    """Jacobi<LAD> (stationary solver / smoother) restated in C."""
    s, T = _sfx(dtype)
    rp, c, v = _csr(rowptr, col, val, T)
    n = rp.shape[0] - 1
    x = np.zeros(n, T) if x0 is None else np.array(x0, T)
    it, res, res0 = C.c_int(), C.c_double(), C.c_double()
    st = getattr(_load(), f"orc_jacobi_{s}")(n, rp, c, v, np.ascontiguousarray(b, T), x, int(mode),
                                             int(maxits), int(inner_iter), int(smooth_iter), float(w),
                                             atol, rtol, dtol, C.byref(it), C.byref(res),
                                             C.byref(res0))
    if st == -2:
        raise ValueError("a row has no nonzero diagonal")
    return OracleResult(x, it.value, res.value, res0.value, st)


def bicgstab(rowptr, col, val, b, x0=None, *, maxits=1000, atol=1e-12, rtol=1e-8, dtol=1e8,
             precond=True, dtype=np.float64) -> tuple[OracleResult, int]:
    """BiCGSTAB<LAD> (no / right Jacobi preconditioning) restated in C.
    Returns the result and the number of restarts."""
    s, T = _sfx(dtype)
    rp, c, v = _csr(rowptr, col, val, T)
    n = rp.shape[0] - 1
    x = np.zeros(n, T) if x0 is None else np.array(x0, T)
    inv = invdiag(rp, c, v, T) if precond else np.zeros(1, T)
    it, rs, res, res0 = C.c_int(), C.c_int(), C.c_double(), C.c_double()
    st = getattr(_load(), f"orc_bicgstab_{s}")(n, rp, c, v, np.ascontiguousarray(b, T), x,
                                               int(bool(precond)), inv, int(maxits), atol, rtol, dtol,
                                               C.byref(it), C.byref(rs), C.byref(res), C.byref(res0))
    return OracleResult(x, it.value, res.value, res0.value, st), rs.value


def gmres(rowptr, col, val, b, x0=None, *, size_basis=100, maxits=1000, atol=1e-12, rtol=1e-8, dtol=1e8,
          precond=True, dtype=np.float64) -> OracleResult:
    """GMRES<LAD> (restarted, modified Gram-Schmidt; no / right Jacobi
    preconditioning) restated in C."""
    s, T = _sfx(dtype)
    rp, c, v = _csr(rowptr, col, val, T)
    n = rp.shape[0] - 1
    x = np.zeros(n, T) if x0 is None else np.array(x0, T)
    inv = invdiag(rp, c, v, T) if precond else np.zeros(1, T)
    it, res, res0 = C.c_int(), C.c_double(), C.c_double()
    st = getattr(_load(), f"orc_gmres_{s}")(n, rp, c, v, np.ascontiguousarray(b, T), x, int(bool(precond)), inv,
                                            int(size_basis), int(maxits), atol, rtol, dtol, C.byref(it),
                                            C.byref(res), C.byref(res0))
    return OracleResult(x, it.value, res.value, res0.value, st)


def ref_gmres(rowptr, col, val, b, x0=None, *, size_basis=100, maxits=1000, atol=1e-12, rtol=1e-8, dtol=1e8,
              precond=True, impl=IMPL_NAIVE, nthreads=1) -> OracleResult:
    """GMRES<LAD> restated over the reference's compiled lmp objects (FP64)."""
    rp, c, v = _csr(rowptr, col, val, np.float64)
    n = rp.shape[0] - 1
    x = np.zeros(n) if x0 is None else np.array(x0, np.float64)
    it, res, res0, sec = C.c_int(), C.c_double(), C.c_double(), C.c_double()
    st = _load_ref().ref_gmres_solve_d(impl, nthreads, int(bool(precond)), n, c.shape[0], rp, c, v,
                                       np.ascontiguousarray(b, np.float64), x, int(size_basis), int(maxits),
                                       atol, rtol, dtol, C.byref(it), C.byref(res), C.byref(res0),
                                       C.byref(sec))
    return OracleResult(x, it.value, res.value, res0.value, st, sec.value)


def coo_to_csr(nrow, ncol, rows, cols, vals):
    """coo_2_csr / TransformFromCOO restated in C: (rowptr, col, val)."""
    rows = np.ascontiguousarray(rows, np.int32)
    cols = np.ascontiguousarray(cols, np.int32)
    vals = np.ascontiguousarray(vals, np.float64)
    nnz = rows.shape[0]
    rp = np.empty(nrow + 1, np.int32)
    c = np.empty(max(nnz, 1), np.int32)
    v = np.empty(max(nnz, 1), np.float64)
    if _load().orc_coo2csr_d(int(nrow), int(ncol), nnz, rows, cols, vals, rp, c, v,
                             np.empty(max(nrow, 1), np.int32)) != 0:
        raise ValueError("COO index out of range")
    return rp, c[:nnz], v[:nnz]


def ref_coo_to_csr(nrow, ncol, rows, cols, vals):
    """The reference's own CPU_CSR_lMatrix::TransformFromCOO: (rowptr, col, val)."""
    rows = np.ascontiguousarray(rows, np.int32)
    cols = np.ascontiguousarray(cols, np.int32)
    vals = np.ascontiguousarray(vals, np.float64)
    nnz = rows.shape[0]
    rp = np.empty(nrow + 1, np.int32)
    c = np.empty(max(nnz, 1), np.int32)
    v = np.empty(max(nnz, 1), np.float64)
    _load_ref().ref_coo_to_csr_d(int(nrow), int(ncol), nnz, rows, cols, vals, rp, c, v)
    return rp, c[:nnz], v[:nnz]


def ref_jacobi(rowptr, col, val, b, x0=None, *, mode=JACOBI_SOLVE_NORMAL, maxits=1000, inner_iter=1,
               smooth_iter=1, w=1.0, atol=1e-12, rtol=1e-8, dtol=1e8, impl=IMPL_NAIVE,
               nthreads=1) -> OracleResult:
    """Jacobi<LAD> restated over the reference's compiled lmp objects (FP64)."""
    rp, c, v = _csr(rowptr, col, val, np.float64)
    n = rp.shape[0] - 1
    x = np.zeros(n) if x0 is None else np.array(x0, np.float64)
    it, res, res0, sec = C.c_int(), C.c_double(), C.c_double(), C.c_double()
    st = _load_ref().ref_jacobi_solve_d(impl, nthreads, int(mode), n, c.shape[0], rp, c, v,
                                        np.ascontiguousarray(b, np.float64), x, int(maxits),
                                        int(inner_iter), int(smooth_iter), float(w), atol, rtol, dtol,
                                        C.byref(it), C.byref(res), C.byref(res0), C.byref(sec))
    return OracleResult(x, it.value, res.value, res0.value, st, sec.value)


def ref_bicgstab(rowptr, col, val, b, x0=None, *, maxits=1000, atol=1e-12, rtol=1e-8, dtol=1e8,
                 precond=True, impl=IMPL_NAIVE, nthreads=1) -> tuple[OracleResult, int]:
    """BiCGSTAB<LAD> restated over the reference's compiled lmp objects (FP64)."""
    rp, c, v = _csr(rowptr, col, val, np.float64)
    n = rp.shape[0] - 1
    x = np.zeros(n) if x0 is None else np.array(x0, np.float64)
    it, rs, res, res0, sec = C.c_int(), C.c_int(), C.c_double(), C.c_double(), C.c_double()
    st = _load_ref().ref_bicgstab_solve_d(impl, nthreads, int(bool(precond)), n, c.shape[0], rp, c, v,
                                          np.ascontiguousarray(b, np.float64), x, int(maxits), atol,
                                          rtol, dtol, C.byref(it), C.byref(rs), C.byref(res),
                                          C.byref(res0), C.byref(sec))
    return OracleResult(x, it.value, res.value, res0.value, st, sec.value), rs.value


def ref_spmv(rowptr, col, val, x, *, impl=IMPL_NAIVE, nthreads=1, dtype=np.float64) -> np.ndarray:
    """CPUsimple/CPUopenmp_CSR_lMatrix::VectorMult from the reference sources."""
    s, T = _sfx(dtype)
    rp, c, v = _csr(rowptr, col, val, T)
    n = rp.shape[0] - 1
    y = np.empty(n, T)
    getattr(_load_ref(), f"ref_spmv_{s}")(impl, nthreads, n, c.shape[0], rp, c, v,
                                          np.ascontiguousarray(x, T), y)
    return y


def ref_cg(rowptr, col, val, b, x0=None, *, maxits=1000, atol=1e-12, rtol=1e-8, dtol=1e8,
           precond=True, impl=IMPL_NAIVE, nthreads=1, dtype=np.float64) -> OracleResult:
    """CG<LAD> restated over the reference's compiled lmp objects."""
    s, T = _sfx(dtype)
    rp, c, v = _csr(rowptr, col, val, T)
    n = rp.shape[0] - 1
    x = np.zeros(n, T) if x0 is None else np.array(x0, T)
    it, res, res0, rel = C.c_int(), C.c_double(), C.c_double(), C.c_double()
    st = getattr(_load_ref(), f"ref_cg_solve_{s}")(
        impl, nthreads, int(bool(precond)), n, c.shape[0], rp, c, v, np.ascontiguousarray(b, T), x,
        int(maxits), atol, rtol, dtol, C.byref(it), C.byref(res), C.byref(res0), C.byref(rel))
    return OracleResult(x, it.value, res.value, res0.value, st)


def ref_lmp_cg(rowptr, col, val, b, x0=None, *, rel_eps=1e-10, abs_eps=0.0, max_iter=10000,
               impl=IMPL_NAIVE, nthreads=1) -> OracleResult:
    """The reference's own lmp cg() (lmp/solvers/cg.cc:35)."""
    rp, c, v = _csr(rowptr, col, val, np.float64)
    n = rp.shape[0] - 1
    x = np.zeros(n) if x0 is None else np.array(x0, np.float64)
    mi = C.c_int(int(max_iter))
    _load_ref().ref_lmp_cg_d(impl, nthreads, n, c.shape[0], rp, c, v,
                             np.ascontiguousarray(b, np.float64), x, rel_eps, abs_eps, C.byref(mi))
    return OracleResult(x, mi.value, float("nan"), float("nan"), 0)


class RefSystem:
    """A matrix built once in the reference's own CPU classes, for timed
    repeated solves (the reported seconds exclude matrix construction)."""

    def __init__(self, rowptr, col, val, *, impl=IMPL_OPENMP, nthreads=None):
        lib = _load_ref()
        lib.ref_system_create.restype = C.c_void_p
        lib.ref_system_create.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, _i32p, _i32p, _f64p]
        lib.ref_system_destroy.argtypes = [C.c_void_p]
        lib.ref_system_cg.argtypes = [C.c_void_p, C.c_int, _f64p, _f64p, C.c_int, C.c_double,
                                      C.c_double, C.c_double, _ip, _dp, _dp, _dp]
        rp, c, v = _csr(rowptr, col, val, np.float64)
        self.n = rp.shape[0] - 1
        self.nthreads = int(nthreads or os.cpu_count() or 1)
        self.impl = impl
        self._lib = lib
        self._h = lib.ref_system_create(impl, self.nthreads, self.n, c.shape[0], rp, c, v)

    def cg(self, b, x0=None, *, maxits=1000, atol=1e-12, rtol=1e-8, dtol=1e8, precond=True):
        x = np.zeros(self.n) if x0 is None else np.array(x0, np.float64)
        it, res, res0, sec = C.c_int(), C.c_double(), C.c_double(), C.c_double()
        st = self._lib.ref_system_cg(self._h, int(bool(precond)), np.ascontiguousarray(b, np.float64), x,
                                     int(maxits), atol, rtol, dtol, C.byref(it), C.byref(res),
                                     C.byref(res0), C.byref(sec))
        return OracleResult(x, it.value, res.value, res0.value, st), sec.value

    def close(self):
        if self._h:
            self._lib.ref_system_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _component(kind, opts, rowptr, col, val, b, x0, maxits, atol, rtol, dtol, dtype):
    """One LinearSolver component of MPIR, solved by the oracle from x0."""
    kw = dict(maxits=maxits, atol=atol, rtol=rtol, dtol=dtol, dtype=dtype)
    if kind == "cg":
        return cg(rowptr, col, val, b, x0, precond=opts.get("precond", True), **kw)
    if kind == "bicgstab":
        return bicgstab(rowptr, col, val, b, x0, precond=opts.get("precond", True), **kw)[0]
    if kind == "gmres":
        return gmres(rowptr, col, val, b, x0, precond=opts.get("precond", True),
                     size_basis=opts.get("size_basis", 100), **kw)
    if kind == "jacobi":
        return jacobi(rowptr, col, val, b, x0, mode=opts.get("mode", 0), inner_iter=opts.get("inner_iter", 1),
                      smooth_iter=opts.get("smooth_iter", 1), w=opts.get("w", 1.0), **kw)
    raise ValueError(kind)


def mpir_generic(rowptr, col, val, b, x0=None, *, max_ech=0, max_ecl=0, abs_tol=0.0, rel_tol=0.0, div_tol=0.0,
                 components=None, use=None):
    """MPIR<LAD_high, LAD_low>::SolveImpl (linear_solver/mpir.cc:52-285) with
    ContinueIteration (:288-297), restated over the oracle's solvers: the
    high-precision parts in float64, the low-precision parts in float32 on
    the float32 copy of the matrix.  components: role -> (kind, options,
    (max_iter, abs_tol, rel_tol, div_tol)) for the roles ech, ecl, preh,
    posth, prel, postl; use: role -> bool for the four smoothers.  As in the
    reference, res0 moves to the latest residual after every pass.  Returns
    a dict with x, res, res_init, iters, n_ecl, n_ech, passes, success."""
    rp, c, v = _csr(rowptr, col, val, np.float64)
    v32 = v.astype(np.float32)
    b = np.ascontiguousarray(b, np.float64)
    n = rp.shape[0] - 1
    x = np.zeros(n) if x0 is None else np.array(x0, np.float64)
    components = components or {}
    use = use or {}
    zero = (0, 0.0, 0.0, 0.0)
    par = {r: (components[r][2] if r in components else zero) for r in ("ech", "ecl", "preh", "posth", "prel",
                                                                          "postl")}
    it = 0
    # Jacobi<LAD> in a smoothing mode never resets iter_ (jacobi.cc:256-285), so
    # the iter() that MPIR adds after each call is that smoother's running total
    smooth_total = {}

    def run(role, bb, xx, low):
        nonlocal it
        kind, opts, (mi, at, rt, dt) = components[role]
        r = _component(kind, opts, rp, c, v32 if low else v, bb, xx, mi, at, rt, dt,
                       np.float32 if low else np.float64)
        if kind == "jacobi" and opts.get("mode", 0) >= 2:
            smooth_total[role] = smooth_total.get(role, 0) + r.iters
            it += smooth_total[role]
        else:
            it += r.iters
        return r.x

    def residual(xx):
        r = b - spmv(rp, c, v, xx)          # VectorMult, ScaleAdd(b, -1): -Ax + b
        return r, float(np.sqrt(dot(r, r)))

    resh, res = residual(x)
    res_init = res0 = res
    n_ech = n_ecl = passes = 0

    def cont():
        pe, ph = par["ecl"], par["ech"]
        return (res > abs_tol and res > res0 * rel_tol and res < div_tol and
                ((n_ech < max_ech and res > ph[1] and res > res0 * ph[2] and res < ph[3]) or
                 (n_ecl < max_ecl and res > pe[1] and res > res0 * pe[2] and res < pe[3])))

    while cont():
        passes += 1
        if use.get("preh"):
            x = run("preh", b, x, False)
            resh, res = residual(x)
        pe, ph = par["ecl"], par["ech"]
        if "ecl" in components and n_ecl < max_ecl and res > pe[1] and res > res0 * pe[2] and res < pe[3]:
            n_ecl += 1
            resl = resh.astype(np.float32)
            corl = np.zeros(n, np.float32)
            if use.get("prel"):
                corl = run("prel", resl, corl, True)
            corl = run("ecl", resl, corl, True)
            if use.get("postl"):
                corl = run("postl", resl, corl, True)
            corh = corl.astype(np.float64)
        elif "ech" in components and n_ech < max_ech and res > ph[1] and res > res0 * ph[2] and res < ph[3]:
            n_ech += 1
            corh = run("ech", resh, np.zeros(n), False)
        x = x + corh
        if use.get("posth"):
            x = run("posth", b, x, False)
        resh, res = residual(x)
        res0 = res
    success = res < abs_tol or res < res0 * rel_tol
    return {"x": x, "res": res, "res_init": res_init, "iters": it, "n_ecl": n_ecl, "n_ech": n_ech,
            "passes": passes, "success": success}
