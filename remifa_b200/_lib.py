"""ctypes binding of liblu_b200.so (the C ABI declared in include/lu_b200.h).

There is no fallback: if the shared library is missing or a call needs a GPU
that is not there, the call raises.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblu_b200.so")

# lu_status
SUCCESS, ERR_INVALID_ARG, ERR_CUDA, ERR_ALLOC, ERR_UNSUPPORTED, ERR_WORKSPACE, \
    ERR_NOT_CONVERGED, ERR_TIMEOUT, ERR_NO_DEVICE = range(9)

# lu_dtype
F32, F16, BF16, E4M3, F64 = range(5)

# lu_compute (0..3 = the reference's remifa::compute_type values)
COMPUTE_FP32, COMPUTE_FP16, COMPUTE_TC32, COMPUTE_TC16, COMPUTE_TC32_BF16, \
    COMPUTE_TC32_E4M3, COMPUTE_TC32_SPLIT = range(7)

RIGHT_LOOKING, LEFT_LOOKING = 0, 1


class LuOpts(ctypes.Structure):
    _fields_ = [
        ("nb", ctypes.c_int64),
        ("ib", ctypes.c_int32),
        ("inner_update", ctypes.c_int32),
        ("outer_update", ctypes.c_int32),
        ("variant", ctypes.c_int32),
        ("lookahead", ctypes.c_int32),
        ("diag_width", ctypes.c_int32),
        ("panel_fp32", ctypes.c_int32),
        ("bulk_steps", ctypes.c_int32),
        ("reserved", ctypes.c_int32 * 6),
    ]


class LuProfileEntry(ctypes.Structure):
    _fields_ = [
        ("name", ctypes.c_char * 32),
        ("launches", ctypes.c_int64),
        ("total_ms", ctypes.c_double),
        ("bytes", ctypes.c_double),
        ("flops", ctypes.c_double),
    ]


BATCH_MAX_N = 512
BATCH_BUCKETS = 6


class LuBatchTuning(ctypes.Structure):
    _fields_ = [
        ("nb", ctypes.c_int32 * BATCH_BUCKETS),
        ("outer", ctypes.c_int32 * BATCH_BUCKETS),
    ]


class LuTraceEntry(ctypes.Structure):
    _fields_ = [
        ("name", ctypes.c_char * 32),
        ("stream", ctypes.c_int32),
        ("start_ms", ctypes.c_double),
        ("end_ms", ctypes.c_double),
    ]


_i64 = ctypes.c_int64
_vp = ctypes.c_void_p
_int = ctypes.c_int

# (name, restype, argtypes) for every entry point of include/lu_b200.h
SIGNATURES = {
    "lu_opts_default": (None, [ctypes.POINTER(LuOpts)]),
    "lu_status_string": (ctypes.c_char_p, [_int]),
    "lu_abi_version": (_int, []),
    "lu_last_error": (ctypes.c_char_p, []),
    "lu_workspace_size": (_int, [ctypes.POINTER(LuOpts), _i64, _i64, _int,
                                 ctypes.POINTER(ctypes.c_size_t)]),
    "lu_nopiv_rl_c": (_int, [ctypes.POINTER(LuOpts), _vp, _i64, _i64, _vp, _int,
                             _i64, _vp, _vp, _i64, _vp, ctypes.c_size_t]),
    "lu_nopiv_rl_host_c": (_int, [ctypes.POINTER(LuOpts), _vp, _i64, _vp, _i64, _vp, _i64,
                                  _vp, _vp, ctypes.c_size_t]),
    "lu_nopiv_ll_c": (_int, [ctypes.POINTER(LuOpts), _vp, _i64, _i64, _vp, _int,
                             _i64, _vp, _vp, _i64, _vp, ctypes.c_size_t]),
    "lu_panel_c": (_int, [_vp, _int, _i64, _i64, _vp, _i64, _vp, _i64, _vp,
                          _i64, _vp]),
    "lu_convert_c": (_int, [_vp, _i64, _i64, _vp, _int, _i64, _vp, _int, _i64,
                            _int]),
    "lu_gemm_update_c": (_int, [_vp, _int, _i64, _i64, _i64, ctypes.c_double,
                                _vp, _i64, _vp, _i64, ctypes.c_double, _vp,
                                _i64, _vp, ctypes.c_size_t]),
    "lu_gemm_update_ex_c": (_int, [_vp, _int, _i64, _i64, _i64, ctypes.c_double,
                                   _vp, _int, _i64, _vp, _int, _i64, ctypes.c_double, _vp,
                                   _int, _i64, _vp, ctypes.c_size_t]),
    "lu_gen_matrix_c": (_int, [_vp, _i64, _vp, _i64, ctypes.c_uint64, _int,
                               ctypes.c_double, _int, ctypes.c_double]),
    "lu_equilibrate_c": (_int, [_vp, _i64, _vp, _i64, _vp, _vp, _int, ctypes.c_char_p,
                                ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                                ctypes.POINTER(ctypes.c_double)]),
    "lu_solve_c": (_int, [_vp, _i64, _vp, _i64, _vp, _i64, _i64, _int]),
    "lu_refine_workspace_size": (_int, [_i64, ctypes.POINTER(ctypes.c_size_t)]),
    "lu_refine_c": (_int, [_vp, _i64, _vp, _i64, _vp, _i64, _vp, _vp, ctypes.c_double,
                           _int, ctypes.POINTER(_int), ctypes.POINTER(ctypes.c_double),
                           _vp, ctypes.c_size_t]),
    "lu_refine_static_c": (_int, [_vp, _i64, _vp, _i64, _vp, _i64, _vp, _vp, ctypes.c_double,
                                  _int, ctypes.POINTER(_int), ctypes.POINTER(ctypes.c_double)]),
    "lu_gmres_ir_workspace_size": (_int, [_i64, _int, ctypes.POINTER(ctypes.c_size_t)]),
    "lu_gmres_ir_c": (_int, [_vp, _i64, _vp, _i64, _vp, _i64, _vp, _vp, ctypes.c_double,
                             _int, _int, ctypes.c_double, ctypes.POINTER(_int),
                             ctypes.POINTER(_int), ctypes.POINTER(ctypes.c_double), _vp,
                             ctypes.c_size_t]),
    "lu_refine_ex_workspace_size": (_int, [_i64, _i64, ctypes.POINTER(ctypes.c_size_t)]),
    "lu_refine_ex_c": (_int, [_vp, _i64, _i64, _vp, _i64, _vp, _i64, _vp, _i64, _vp,
                              _i64, _int, ctypes.c_double, _int, ctypes.POINTER(_int),
                              ctypes.POINTER(ctypes.c_double), _vp, ctypes.c_size_t]),
    "lu_adjoint_workspace_size": (_int, [_i64, _i64, ctypes.POINTER(ctypes.c_size_t)]),
    "lu_adjoint_c": (_int, [_vp, _i64, _i64, _vp, _i64, _vp, _i64, _vp, _i64, _vp, _i64,
                            _vp, _i64, ctypes.c_double, _int, ctypes.POINTER(_int),
                            ctypes.POINTER(ctypes.c_double), _vp, ctypes.c_size_t]),
    "lu_batch_plan_create": (_int, [ctypes.POINTER(LuOpts), _i64, _vp,
                                    ctypes.POINTER(LuBatchTuning), ctypes.POINTER(_vp)]),
    "lu_batch_plan_destroy": (None, [_vp]),
    "lu_batch_plan_tuning": (_int, [_vp, ctypes.POINTER(LuBatchTuning)]),
    "lu_batch_plan_set_tuning": (_int, [_vp, ctypes.POINTER(LuBatchTuning)]),
    "lu_batch_c": (_int, [_vp, _vp, _vp, _vp, _vp]),
    "lu_batch_autotune": (_int, [_vp, _vp, _int, ctypes.POINTER(LuBatchTuning)]),
    "lu_batch_graph_create": (_int, [_vp, _vp, _vp, _vp, _vp, ctypes.POINTER(_vp)]),
    "lu_batch_graph_launch": (_int, [_vp, _vp]),
    "lu_batch_graph_destroy": (None, [_vp]),
    "lu_batch_solve_c": (_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, ctypes.c_int32, _int,
                                _int]),
    "lu_batch_adjoint_c": (_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                  ctypes.c_int32, _int]),
    "lu_gen_batch_c": (_int, [_vp, _i64, _vp, _vp, _vp, ctypes.c_uint64, _int,
                              ctypes.c_double]),
    "lu_selfcheck_rcp_c": (_int, [_vp, _vp]),
    "lu_selftest_wait_update_c": (_int, [_vp, ctypes.c_longlong, _int, _vp, ctypes.c_size_t,
                                         _vp]),
    "lu_selftest_wait_solve_c": (_int, [_vp, ctypes.c_ulonglong, _i64, _vp, _i64, _vp, _vp,
                                        ctypes.c_size_t, _vp]),
    "lu_catchup_row_step_c": (_int, [_vp, _int, _int, _i64, _i64, _i64, _i64, _vp, _i64, _vp,
                                     _i64, _vp, _vp, _i64, _vp, _i64, _i64, _int, _vp]),
    "lu_profile_begin": (None, []),
    "lu_profile_end": (_int, [ctypes.POINTER(LuProfileEntry), _int]),
    "lu_launch_count": (ctypes.c_longlong, []),
    "lu_trim_memory_c": (_int, []),
    "lu_profile_trace": (_int, [ctypes.POINTER(LuTraceEntry), _int]),
}

_lib = None


def lib() -> ctypes.CDLL:
    """Load liblu_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m remifa_b200.build`"
            )
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


class LuError(RuntimeError):
    def __init__(self, status: int, where: str):
        L = lib()
        msg = L.lu_status_string(status).decode()
        detail = L.lu_last_error().decode()
        super().__init__(f"{where}: {msg}" + (f" [{detail}]" if detail else ""))
        self.status = status


def check(status: int, where: str) -> None:
    """Map an lu_status to the reference's error behaviour: invalid
    arguments raise ValueError (the reference throws std::invalid_argument),
    unsupported combinations raise NotImplementedError (the reference prints
    and exits), everything else raises LuError (std::runtime_error)."""
    if status == SUCCESS:
        return
    if status == ERR_INVALID_ARG:
        raise ValueError(f"{where}: invalid argument")
    if status == ERR_UNSUPPORTED:
        raise NotImplementedError(f"{where}: unsupported combination")
    raise LuError(status, where)
