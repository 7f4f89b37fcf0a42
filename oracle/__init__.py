"""TEST INFRASTRUCTURE ONLY: numpy bindings to the CPU oracle (liboracle.so).

The oracle restates the reference no-pivot LU (flipflapflop/remifa
``src/lu_nopiv.hxx``, ``src/lu_nopiv_inner_rl.hxx``, ``src/lu_nopiv.cu``,
``src/convert.cu``) on the CPU with an explicit floating-point order, plus an
FP64 factorization, the reference's error formulas (``tests/errors.hxx``) and
its matrix generators (``tests/genmat.hxx``, ``tests/common.hxx``).

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package; the product library never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_REF_PATH = os.path.join(_HERE, "_ref", "libremifa_ref.so")

_i64 = ctypes.c_int64
_f32p = ctypes.POINTER(ctypes.c_float)
_f64p = ctypes.POINTER(ctypes.c_double)

FMT_FP32, FMT_FP16, FMT_BF16, FMT_E4M3, FMT_SPLIT = 0, 1, 2, 3, 4


def build(force: bool = False) -> None:
    """Compile liboracle.so with the committed Makefile."""
    if force or not os.path.exists(_LIB_PATH):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)


def build_ref() -> bool:
    """Compile the reference's GPU sources into _ref/ (needs the reference
    tree, present only in the development container).  Returns success."""
    ref = os.environ.get("REMIFA_REF_DIR", "/root/reference")
    if not os.path.isdir(os.path.join(ref, "src")):
        return os.path.exists(_REF_PATH)
    subprocess.run(["make", "-s", "-C", _HERE, "ref", f"REF={ref}"], check=True)
    return True


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        L.orc_gen_diagdom_f32.argtypes = [_i64, _i64, _f32p, _i64]
        L.orc_gen_randmat_f32.argtypes = [_i64, _i64, _f32p, _i64, ctypes.c_uint32]
        L.orc_gen_matrix_f32.argtypes = [_i64, _f32p, _i64, ctypes.c_uint64,
                                         ctypes.c_int, ctypes.c_double,
                                         ctypes.c_int, ctypes.c_double]
        L.orc_gen_vector_f64.argtypes = [_i64, _f64p, ctypes.c_uint64, ctypes.c_int]
        L.orc_gen_rhs_f32.argtypes = [_i64, _f32p, _i64, _f32p, _f32p]
        L.orc_round_fmt.argtypes = [ctypes.c_float, ctypes.c_int, ctypes.c_int]
        L.orc_round_fmt.restype = ctypes.c_float
        L.orc_convert.argtypes = [_i64, _i64, _f32p, _i64, _f32p, _i64,
                                  ctypes.c_int, ctypes.c_int]
        L.orc_panel_f32.argtypes = [_i64, _i64, _f32p, _i64, _f32p, _i64, _f32p, _i64]
        L.orc_panel_f16.argtypes = [_i64, _i64, _f32p, _i64, _f32p, _i64, _f32p, _i64]
        L.orc_gemm_sub_f32.argtypes = [_i64, _i64, _i64, _f32p, _i64, _f32p,
                                       _i64, _f32p, _i64]
        L.orc_lu_rl_f32.argtypes = [_i64, _i64, _i64, _f32p, _i64, ctypes.c_int,
                                    ctypes.c_int]
        L.orc_lu_rl_f32_range.argtypes = [_i64, _i64, _i64, _f32p, _i64, ctypes.c_int,
                                          ctypes.c_int, _i64, _i64]
        L.orc_lu_ll_f32.argtypes = [_i64, _i64, _i64, _f32p, _i64, ctypes.c_int]
        L.orc_lu_ll_f16.argtypes = [_i64, _i64, _i64, _f32p, _i64, ctypes.c_int]
        L.orc_lu_ll_f32_sub.argtypes = [_i64, _i64, _i64, _f32p, _i64, ctypes.c_int, _i64]
        L.orc_lu_ll_f16_ex.argtypes = [_i64, _i64, _i64, _f32p, _i64, ctypes.c_int, _i64,
                                       ctypes.c_int]
        L.orc_lu_f64.argtypes = [_i64, _f64p, _i64]
        L.orc_lu_solve_f64.argtypes = [_i64, _f64p, _i64, _f64p]
        L.orc_lu_solve_f32.argtypes = [_i64, _f32p, _i64, _f32p]
        L.orc_lu_solve_f32f64.argtypes = [_i64, _f32p, _i64, _f64p]
        L.orc_nwerr_f32.argtypes = [_i64, _f32p, _i64, _f32p, _f32p]
        L.orc_nwerr_f32.restype = ctypes.c_double
        L.orc_cwerr_f32.argtypes = [_i64, _f32p, _i64, _f32p, _f32p, _f32p, _i64]
        L.orc_cwerr_f32.restype = ctypes.c_double
        L.orc_factor_error_f32.argtypes = [_i64, _f32p, _i64, _f32p, _i64]
        L.orc_factor_error_f32.restype = ctypes.c_double
        L.orc_backward_error_f64.argtypes = [_i64, _f32p, _i64, _f64p, _f64p]
        L.orc_backward_error_f64.restype = ctypes.c_double
        L.orc_num_threads.restype = ctypes.c_int
        _lib = L
    return _lib


def _p32(a: np.ndarray):
    assert a.dtype == np.float32
    return a.ctypes.data_as(_f32p)


def _p64(a: np.ndarray):
    assert a.dtype == np.float64
    return a.ctypes.data_as(_f64p)


def colmajor(m: int, n: int, lda: int | None = None, dtype=np.float32) -> np.ndarray:
    """A column-major m x n array with leading dimension lda (a Fortran-ordered
    view into an lda x n buffer)."""
    lda = m if lda is None else lda
    buf = np.zeros((n, lda), dtype=dtype)
    return buf.T[:m, :]


def ld(a: np.ndarray) -> int:
    """Leading dimension of a Fortran-ordered (column-major) view."""
    return a.strides[1] // a.itemsize


def gen_diagdom(m: int, lda: int | None = None) -> np.ndarray:
    a = colmajor(m, m, lda)
    lib().orc_gen_diagdom_f32(m, m, _p32(a), ld(a))
    return a


def gen_randmat(m: int, seed: int = 1, lda: int | None = None) -> np.ndarray:
    a = colmajor(m, m, lda)
    lib().orc_gen_randmat_f32(m, m, _p32(a), ld(a), seed)
    return a


def gen_matrix(n: int, seed: int, kind: int = 0, alpha: float = 2.0,
               kscale: int = 0, gamma_bits: float = 0.0,
               lda: int | None = None) -> np.ndarray:
    a = colmajor(n, n, lda)
    lib().orc_gen_matrix_f32(n, _p32(a), ld(a), seed, kind, alpha, kscale,
                             gamma_bits)
    return a


def gen_vector(n: int, seed: int, kind: int = 1) -> np.ndarray:
    x = np.zeros(n, dtype=np.float64)
    lib().orc_gen_vector_f64(n, _p64(x), seed, kind)
    return x


def gen_rhs(a: np.ndarray, x: np.ndarray) -> np.ndarray:
    m = a.shape[0]
    x = np.ascontiguousarray(x, dtype=np.float32)
    b = np.zeros(m, dtype=np.float32)
    lib().orc_gen_rhs_f32(m, _p32(a), ld(a), _p32(x), _p32(b))
    return b


def round_fmt(a: np.ndarray, fmt: int, scale_log2: int = 0) -> np.ndarray:
    a = np.asfortranarray(a, dtype=np.float32)
    out = colmajor(a.shape[0], a.shape[1])
    lib().orc_convert(a.shape[0], a.shape[1], _p32(a), ld(a), _p32(out), ld(out),
                      fmt, scale_log2)
    return out


def panel(m: int, n: int, d: np.ndarray, a: np.ndarray) -> None:
    """In place on the block column a (m x >=m for the U part)."""
    lib().orc_panel_f32(m, n, _p32(d), ld(d), _p32(a), ld(a), _p32(a), ld(a))


def panel_f16(m: int, n: int, d: np.ndarray, a: np.ndarray) -> None:
    """lu_nopiv_panel<half,8> restated: in place on the block column a
    (float32 holding fp16 values)."""
    lib().orc_panel_f16(m, n, _p32(d), ld(d), _p32(a), ld(a), _p32(a), ld(a))


def gemm_sub(a: np.ndarray, b: np.ndarray, c: np.ndarray) -> None:
    m, k = a.shape
    n = b.shape[1]
    lib().orc_gemm_sub_f32(m, n, k, _p32(a), ld(a), _p32(b), ld(b), _p32(c), ld(c))


def lu_rl(a: np.ndarray, nb: int = 256, outer_fmt: int = 0, threads: int = 0) -> np.ndarray:
    """Factor a copy of `a` with the restated reference RL algorithm."""
    lda = ld(a) if a.strides[0] == a.itemsize else a.shape[0]
    out = colmajor(a.shape[0], a.shape[1], lda)
    out[:, :] = a
    lib().orc_lu_rl_f32(a.shape[0], a.shape[1], nb, _p32(out), ld(out), outer_fmt, threads)
    return out


def lu_ll(a: np.ndarray, nb: int = 256, threads: int = 0,
          fp16_storage: bool = False, panel_fp32: bool = False,
          sub: int = 128) -> np.ndarray:
    """Factor a copy of `a` with the restated reference left-looking
    algorithm (fp16_storage: the fp16-matrix variant; `a` must then hold
    fp16-representable values; panel_fp32: its OP = OF = fp32 form).  Outer
    blocks wider than `sub` are factored as sub-blocks of that width, as the
    product library does (for nb <= sub this is the reference's loop)."""
    lda = ld(a) if a.strides[0] == a.itemsize else a.shape[0]
    out = colmajor(a.shape[0], a.shape[1], lda)
    out[:, :] = a
    if fp16_storage:
        lib().orc_lu_ll_f16_ex(a.shape[0], a.shape[1], nb, _p32(out), ld(out), threads,
                               sub, int(bool(panel_fp32)))
    else:
        lib().orc_lu_ll_f32_sub(a.shape[0], a.shape[1], nb, _p32(out), ld(out), threads,
                                sub)
    return out


def lu_rl_steps(a: np.ndarray, nb: int, outer_fmt: int, kk0: int, kk1: int,
                threads: int = 0) -> None:
    """In place: outer steps [kk0, kk1) of the restated RL factorization."""
    lib().orc_lu_rl_f32_range(a.shape[0], a.shape[1], nb, _p32(a), ld(a), outer_fmt,
                              threads, kk0, kk1)


def lu_f64(a: np.ndarray) -> np.ndarray:
    out = np.asfortranarray(a, dtype=np.float64).copy(order="F")
    lib().orc_lu_f64(out.shape[0], _p64(out), ld(out))
    return out


def lu_solve_f64(lu: np.ndarray, b: np.ndarray) -> np.ndarray:
    x = np.array(b, dtype=np.float64, copy=True)
    if lu.dtype == np.float32:
        lib().orc_lu_solve_f32f64(lu.shape[0], _p32(lu), ld(lu), _p64(x))
    else:
        lib().orc_lu_solve_f64(lu.shape[0], _p64(lu), ld(lu), _p64(x))
    return x


def lu_solve_f32(lu: np.ndarray, b: np.ndarray) -> np.ndarray:
    x = np.array(b, dtype=np.float32, copy=True)
    lib().orc_lu_solve_f32(lu.shape[0], _p32(lu), ld(lu), _p32(x))
    return x


def nwerr(a: np.ndarray, b: np.ndarray, x: np.ndarray) -> float:
    b = np.ascontiguousarray(b, dtype=np.float32)
    x = np.ascontiguousarray(x, dtype=np.float32)
    return lib().orc_nwerr_f32(a.shape[0], _p32(a), ld(a), _p32(b), _p32(x))


def cwerr(a: np.ndarray, b: np.ndarray, x: np.ndarray, lu: np.ndarray) -> float:
    b = np.ascontiguousarray(b, dtype=np.float32)
    x = np.ascontiguousarray(x, dtype=np.float32)
    return lib().orc_cwerr_f32(a.shape[0], _p32(a), ld(a), _p32(b), _p32(x),
                               _p32(lu), ld(lu))


def factor_error(a: np.ndarray, lu: np.ndarray) -> float:
    return lib().orc_factor_error_f32(a.shape[0], _p32(a), ld(a), _p32(lu), ld(lu))


def backward_error(a: np.ndarray, b: np.ndarray, x: np.ndarray) -> float:
    b = np.ascontiguousarray(b, dtype=np.float64)
    x = np.ascontiguousarray(x, dtype=np.float64)
    return lib().orc_backward_error_f64(a.shape[0], _p32(a), ld(a), _p64(b), _p64(x))


def num_threads() -> int:
    return lib().orc_num_threads()
