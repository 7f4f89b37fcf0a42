"""remifa_b200: B200-native (sm_100a) no-pivot LU factorization.

A drop-in for the lu_nopiv entry points of flipflapflop/remifa.  The compute
lives in liblu_b200.so (hand-written CUDA for sm_100a behind the C ABI in
include/lu_b200.h); this package is the thin Python host layer over it.
"""
from . import _lib
from . import batch
from .api import (FP16, FP32, TC16, TC32, align_lda, colmajor, colmajor_empty,
                  compute_type, convert, equilibrate, gemmex, gen_matrix, gesv_mixed, gmres_ir,
                  launch_count, ld, lu_nopiv_ll, lu_nopiv_panel, lu_nopiv_rl, lu_nopiv_rl_host,
                  lu_solve, make_opts, profile, refine, trim_memory, workspace_size)

__all__ = [
    "FP16", "FP32", "TC16", "TC32", "align_lda", "colmajor", "colmajor_empty",
    "compute_type", "convert", "gemmex", "gen_matrix", "ld", "lu_nopiv_ll",
    "lu_nopiv_panel", "lu_nopiv_rl", "lu_nopiv_rl_host", "make_opts", "workspace_size", "profile",
    "launch_count", "lu_solve", "refine", "gesv_mixed", "gmres_ir", "equilibrate",
    "trim_memory",
]


def library_path() -> str:
    return _lib.LIB_PATH
