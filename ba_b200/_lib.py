"""ctypes binding of libb200la.so (the C ABI in include/b200la.h).

The library is the product path: there is no CPU fallback.  Loading fails
loudly when the shared library is missing, and every non-zero status becomes
a B200LAError carrying the library's message.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libb200la.so")

F64, F32 = 0, 1
FMT_CSR, FMT_SELL, FMT_SELL16, FMT_STENCIL = 1, 4, 5, 6
FORMAT_NAMES = {FMT_CSR: "csr", FMT_SELL: "sell", FMT_SELL16: "sell16", FMT_STENCIL: "stencil"}
ITERATE, SUCCESS_ABS, SUCCESS_REL, FAIL_DIV, FAIL_MAXITS, FAIL_BREAKDOWN, DONE_FIXED = range(7)
METHOD_JACOBI, METHOD_BICGSTAB, METHOD_GMRES = 1, 2, 3
SOLVER_SUCCESS, SOLVER_EXCEEDED, SOLVER_ERROR = range(3)
STATUS_NAMES = {0: "OK", -1: "ERR_INVALID", -2: "ERR_CUDA", -3: "ERR_NOMEM", -4: "ERR_DTYPE",
                -5: "ERR_MATRIX", -6: "ERR_TIMEOUT", -7: "ERR_UNSUPPORTED"}


class B200LAError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"b200la {STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class CgParams(C.Structure):
    _fields_ = [("maxits", C.c_int), ("atol", C.c_double), ("rtol", C.c_double),
                ("dtol", C.c_double), ("precond", C.c_int), ("stop_rule", C.c_int)]


class MpParams(C.Structure):
    _fields_ = [("max_outer", C.c_int), ("atol", C.c_double), ("rtol", C.c_double),
                ("dtol", C.c_double), ("inner_maxits", C.c_int), ("inner_rtol", C.c_double),
                ("precond", C.c_int), ("tune", C.c_int), ("inner_storage", C.c_int),
                ("restart_inner", C.c_int)]


class MpResult(C.Structure):
    _fields_ = [("outer", C.c_int), ("inner_iters", C.c_int), ("state", C.c_int),
                ("solver_state", C.c_int), ("res", C.c_double), ("res_init", C.c_double),
                ("res_rel", C.c_double)]


class BatchParams(C.Structure):
    _fields_ = [("capacity", C.c_int), ("mixed", C.c_int), ("precond", C.c_int), ("max_outer", C.c_int),
                ("inner_maxits", C.c_int), ("adaptive", C.c_int), ("tile_rows", C.c_int), ("index_bits", C.c_int),
                ("atol", C.c_double), ("rtol", C.c_double), ("dtol", C.c_double), ("inner_rtol", C.c_double),
                ("restart_inner", C.c_int)]


class SysResult(C.Structure):
    _fields_ = [("state", C.c_int), ("solver_state", C.c_int), ("iters", C.c_int), ("outer", C.c_int),
                ("phase_done", C.c_int), ("reserved", C.c_int), ("res", C.c_double), ("res_init", C.c_double),
                ("res_rel", C.c_double), ("device_us", C.c_double)]


class ServerParams(C.Structure):
    _fields_ = [("batch", BatchParams), ("hbm_budget", C.c_int64), ("chunk_passes", C.c_int),
                ("max_skips", C.c_int)]


class ServerStats(C.Structure):
    _fields_ = [(k, C.c_int64) for k in ("submitted", "completed", "failed", "running", "queued",
                                         "hbm_in_use", "hbm_peak", "hbm_budget", "launches", "passes")] + \
               [(k, C.c_double) for k in ("p50_ms", "p99_ms", "mean_ms", "max_ms", "solves_per_s", "wall_s")]


class CgResult(C.Structure):
    _fields_ = [("iters", C.c_int), ("state", C.c_int), ("solver_state", C.c_int),
                ("reserved", C.c_int), ("res", C.c_double), ("res_init", C.c_double),
                ("res_rel", C.c_double)]


class SolverParams(C.Structure):
    _fields_ = [("method", C.c_int), ("maxits", C.c_int), ("atol", C.c_double), ("rtol", C.c_double),
                ("dtol", C.c_double), ("precond", C.c_int), ("mode", C.c_int), ("inner_iter", C.c_int),
                ("smooth_iter", C.c_int), ("w", C.c_double), ("size_basis", C.c_int)]


class SolverResult(C.Structure):
    _fields_ = [("iters", C.c_int), ("state", C.c_int), ("solver_state", C.c_int),
                ("restarts", C.c_int), ("res", C.c_double), ("res_init", C.c_double),
                ("res_rel", C.c_double)]


_vp = C.c_void_p
_i = C.c_int
_i64 = C.c_int64
_d = C.c_double
_P = C.POINTER

# name -> argtypes (all return int unless listed in _RESTYPE)
_SIGS = {
    "b200la_version": [],
    "b200la_last_error": [],
    "b200la_ctx_create": [_i, _P(_vp)],
    "b200la_ctx_destroy": [_vp],
    "b200la_ctx_set_stream": [_vp, _vp],
    "b200la_ctx_get_stream": [_vp, _P(_vp)],
    "b200la_ctx_synchronize": [_vp],
    "b200la_ctx_set_graphs": [_vp, _i],
    "b200la_ctx_num_sms": [_vp, _P(_i)],
    "b200la_vec_create": [_vp, _i64, _i, _P(_vp)],
    "b200la_vec_wrap": [_vp, _i64, _i, _vp, _P(_vp)],
    "b200la_vec_destroy": [_vp],
    "b200la_vec_info": [_vp, _P(_i64), _P(_i), _P(_vp)],
    "b200la_vec_upload": [_vp, _vp, _i64],
    "b200la_vec_download": [_vp, _vp, _i64],
    "b200la_vec_set_values": [_vp, _vp, _vp, _i],
    "b200la_vec_get_values": [_vp, _vp, _vp, _i],
    "b200la_vec_zeros": [_vp],
    "b200la_vec_copy": [_vp, _vp],
    "b200la_vec_cast": [_vp, _vp],
    "b200la_vec_dot": [_vp, _vp, _P(_d)],
    "b200la_vec_norm2": [_vp, _P(_d)],
    "b200la_vec_axpy": [_vp, _vp, _d],
    "b200la_vec_scaleadd": [_vp, _d, _vp],
    "b200la_vec_scale": [_vp, _d],
    "b200la_vec_elementwise_mult": [_vp, _vp],
    "b200la_vec_range_update": [_vp, _i64, _vp, _i64, _i64, _i, _d],
    "b200la_vec_gather": [_vp, _vp, _i64, _vp],
    "b200la_vec_scatter": [_vp, _vp, _i64, _vp],
    "b200la_dot_noalloc": [_vp, _vp, _i64, _i, _vp, _P(_d)],
    "b200la_csr_upload": [_vp, _i, _i, _i64, _vp, _vp, _vp, _i, _i, _P(_vp)],
    "b200la_coo_upload": [_vp, _i, _i, _i64, _vp, _vp, _vp, _i, _i, _i, _P(_vp)],
    "b200la_mat_download": [_vp, _vp, _vp, _vp],
    "b200la_mat_destroy": [_vp],
    "b200la_mat_info": [_vp, _P(_i), _P(_i), _P(_i64), _P(_i)],
    "b200la_mat_cast": [_vp, _i, _P(_vp)],
    "b200la_mat_zero_rows": [_vp, _vp, _i, _d],
    "b200la_spmv": [_vp, _vp, _vp],
    "b200la_spmv_add": [_vp, _vp, _vp],
    "b200la_spmv_nodiag": [_vp, _vp, _vp],
    "b200la_mat_inv_diag": [_vp, _vp],
    "b200la_mat_set_format": [_vp, _i, _i],
    "b200la_mat_get_format": [_vp, _P(_i), _P(_i)],
    "b200la_mat_to_sell": [_vp, _i, _i, _i, _i],
    "b200la_mat_get_sell": [_vp, _P(_i), _P(_i), _P(_i64)],
    "b200la_mat_tune": [_vp, _P(_i), _P(_i), _P(_d)],
    "b200la_cg_create": [_vp, _P(CgParams), _P(_vp)],
    "b200la_cg_destroy": [_vp],
    "b200la_cg_solve": [_vp, _vp, _vp, _P(CgResult)],
    "b200la_cg_profile": [_vp, _vp, _vp, _i, _P(_d)],
    "b200la_pcg_solve": [_vp, _vp, _vp, _P(CgParams), _P(CgResult)],
    "b200la_solver_create": [_vp, _P(SolverParams), _P(_vp)],
    "b200la_solver_destroy": [_vp],
    "b200la_solver_solve": [_vp, _vp, _vp, _P(SolverResult)],
    "b200la_solver_profile": [_vp, _vp, _vp, _i, _P(_d)],
    "b200la_batch_create": [_vp, _P(BatchParams), _P(_vp)],
    "b200la_batch_destroy": [_vp],
    "b200la_batch_slot_bytes": [_i64, _i64, _i, _i, _P(_i64)],
    "b200la_batch_add": [_vp, _i, _i64, _vp, _vp, _vp, _vp, _vp, _P(_i)],
    "b200la_batch_remove": [_vp, _i],
    "b200la_batch_launch": [_vp, _i],
    "b200la_batch_set_outputs": [_vp, _i, _P(_i), _P(_vp)],
    "b200la_batch_remove_many": [_vp, _i, _P(_i)],
    "b200la_batch_run": [_vp, _i, _P(_i)],
    "b200la_batch_result": [_vp, _i, _vp, _P(SysResult)],
    "b200la_batch_results": [_vp, _i, _P(_i), _P(_vp), _P(SysResult)],
    "b200la_batch_info": [_vp, _P(_i), _P(_i64)],
    "b200la_batch_tune": [_vp, _P(_i), _P(_d)],
    "b200la_batch_set_items": [_vp, _i, _i, _i, _i],
    "b200la_batch_get_items": [_vp, _P(_i)],
    "b200la_batch_restart": [_vp],
    "b200la_batch_last_run": [_vp, _P(_i), _P(_d)],
    "b200la_batch_solve": [_vp, _i, _P(_i)],
    "b200la_batch_profile": [_vp, _i, _P(_d), _P(_i64)],
    "b200la_batch_profile_pass": [_vp, _i, _P(_d), _P(_i64)],
    "b200la_batch_add_q1": [_vp, _i, _i, C.c_uint64, _d, _P(_i)],
    "b200la_batch_add_many": [_vp, _i, _P(_i), _P(_i64), _P(_vp), _P(_vp), _P(_vp), _P(_vp), _P(_vp), _P(_i), _P(_i)],
    "b200la_batch_get_system": [_vp, _i, _vp, _vp, _vp, _vp],
    "b200la_batch_slot_size": [_vp, _i, _P(_i), _P(_i64)],
    "b200la_server_start": [_vp, _P(ServerParams), _P(_vp)],
    "b200la_server_stop": [_vp],
    "b200la_server_submit_csr": [_vp, _i, _i64, _vp, _vp, _vp, _vp, _vp, _P(_i64)],
    "b200la_server_submit_q1": [_vp, _i, _i, C.c_uint64, _d, _P(_i64)],
    "b200la_server_poll": [_vp, _i64, _P(_i), _vp, _P(SysResult), _P(_d)],
    "b200la_server_wait": [_vp, _i64, _d, _P(_i)],
    "b200la_server_release": [_vp, _i64],
    "b200la_server_drain": [_vp, _d],
    "b200la_server_get_stats": [_vp, _P(ServerStats)],
    "b200la_server_reset_stats": [_vp],
    "b200la_q1_size": [_i, _i, _P(_i64), _P(_i64)],
    "b200la_q1_assemble": [_vp, _i, _i, C.c_uint64, _d, _vp, _vp, _vp, _vp],
    "b200la_mp_create": [_vp, _P(MpParams), _P(_vp)],
    "b200la_mp_destroy": [_vp],
    "b200la_mp_inner_matrix": [_vp, _P(_vp)],
    "b200la_mp_solve": [_vp, _vp, _vp, _P(MpResult)],
}
_RESTYPE = {"b200la_version": C.c_char_p, "b200la_last_error": C.c_char_p}

_lib = None


def load():
    """Load libb200la.so once; raise if it is missing (no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C ba_b200/csrc` "
                           "(or __graft_entry__.build())")
    lib = C.CDLL(LIB_PATH)
    for name, args in _SIGS.items():
        fn = getattr(lib, name, None)
        if fn is None:
            continue
        fn.argtypes = args
        fn.restype = _RESTYPE.get(name, C.c_int)
    _lib = lib
    return lib


def exported_symbols() -> list[str]:
    return list(_SIGS)


def check(status: int) -> None:
    if status != 0:
        msg = load().b200la_last_error()
        raise B200LAError(status, msg.decode() if msg else "")


def call(name: str, *args) -> None:
    check(getattr(load(), name)(*args))
