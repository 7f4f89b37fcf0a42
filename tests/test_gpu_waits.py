"""The give-up path of the bounded device waits, made to run out on purpose
and by construction (no fault, no hang): the tensor-core update with its TMA
producer withheld, and the triangular solve with the row block solved first
withholding its solution, each with a short bound.  Afterwards the context
must still be usable: a normal factorization and solve run and are right."""
import ctypes

import numpy as np
import pytest
import torch

import oracle as O
import remifa_b200 as rb
from remifa_b200 import _lib

pytestmark = pytest.mark.gpu
SCRATCH = 2 << 20  # LU_SELFTEST_SCRATCH_BYTES


def _st():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _context_still_usable():
    n = 512
    a = O.gen_matrix(n, seed=3, kind=1, alpha=1.5)
    d = rb.colmajor(torch.from_numpy(a).cuda())
    info = rb.lu_nopiv_rl(d, nb=128, outer=rb.TC32)
    torch.cuda.synchronize()
    assert int(info.item()) == 0
    want = O.lu_rl(a, nb=128, outer_fmt=O.FMT_FP16)
    got = np.asfortranarray(d.cpu().numpy())
    assert np.abs(got - want).max() / np.abs(want).max() < 64 * n * 2.0 ** -24


@pytest.mark.parametrize("streaming", [0, 1])
def test_update_wait_gives_up_and_reports_timeout(built, streaming):
    """~20 us bound (40k cycles at 2 GHz) instead of ~2 s: the MMA warp's
    and the epilogue's waits run out, the kernel records its code and
    returns, and the factorization-level info is -1 (LU_ERR_TIMEOUT)."""
    scratch = torch.empty(SCRATCH, dtype=torch.uint8, device="cuda")
    out = torch.full((2,), 12345, dtype=torch.int32, device="cuda")
    st = _lib.lib().lu_selftest_wait_update_c(_st(), 40_000, streaming,
                                              ctypes.c_void_p(scratch.data_ptr()),
                                              SCRATCH, ctypes.c_void_p(out.data_ptr()))
    assert st == _lib.SUCCESS
    torch.cuda.synchronize()
    code, info = [int(v) for v in out.cpu()]
    assert code in (1, 3), code   # kErrTimeoutFull (MMA warp) / kErrTimeoutTmemFull
    assert info == -1
    _context_still_usable()


def test_solve_wait_gives_up_with_nan(built):
    n = 512
    lu = rb.colmajor(torch.eye(n, dtype=torch.float32, device="cuda"))
    x = torch.ones(n, dtype=torch.float64, device="cuda")
    scratch = torch.empty(1 << 16, dtype=torch.uint8, device="cuda")
    expired = torch.zeros(1, dtype=torch.int32, device="cuda")
    st = _lib.lib().lu_selftest_wait_solve_c(_st(), 20_000, n, ctypes.c_void_p(lu.data_ptr()),
                                             n, ctypes.c_void_p(x.data_ptr()),
                                             ctypes.c_void_p(scratch.data_ptr()),
                                             scratch.numel(),
                                             ctypes.c_void_p(expired.data_ptr()))
    assert st == _lib.SUCCESS
    torch.cuda.synchronize()
    xs = x.cpu().numpy()
    assert np.isnan(xs).all()       # no block after the withheld one looks solved
    assert int(expired.item()) >= 1
    # the same solve without withholding: x = b for the identity factors
    y = torch.ones(n, dtype=torch.float64, device="cuda")
    rb.lu_solve(lu, y)
    torch.cuda.synchronize()
    assert torch.equal(y, torch.ones_like(y))
    _context_still_usable()


def test_selftest_argument_checks(built):
    L = _lib.lib()
    assert L.lu_selftest_wait_update_c(None, 0, 0, ctypes.c_void_p(1024), SCRATCH,
                                       ctypes.c_void_p(64)) == _lib.ERR_INVALID_ARG
    assert L.lu_selftest_wait_solve_c(None, 0, 512, ctypes.c_void_p(64), 512,
                                      ctypes.c_void_p(64), ctypes.c_void_p(64), 1 << 16,
                                      ctypes.c_void_p(64)) == _lib.ERR_INVALID_ARG
