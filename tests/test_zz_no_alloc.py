"""lu_refine_static_c (refinement with compiled-in scratch, no allocation)
against lu_refine_c on the same inputs.  Kept in its own file, collected
last, so it also runs after every other test has used the device."""
import ctypes

import numpy as np
import pytest
import torch

import oracle as O
import remifa_b200 as rb
from remifa_b200 import _lib


def test_static_rejects_n_above_limit():
    """Rejected before any device work (runs without a GPU)."""
    L = _lib.lib()
    st = L.lu_refine_static_c(None, 4097, None, 4097, None, 4097, None, None,
                              1e-14, 30, None, None)
    assert st == _lib.ERR_INVALID_ARG
    assert b"LU_REFINE_STATIC_MAX_N" in L.lu_last_error()
    need = ctypes.c_size_t(0)
    assert L.lu_refine_workspace_size(4096, ctypes.byref(need)) == _lib.SUCCESS
    assert need.value <= 614400   # LU_REFINE_STATIC_SCRATCH_BYTES


@pytest.mark.gpu
@pytest.mark.parametrize("n,outer", [(1000, rb.TC32), (4096, rb.TC32), (257, rb.FP32)])
def test_static_matches_workspace_path_twice(built, n, outer):
    a = O.gen_matrix(n, seed=21, kind=1, alpha=1.5)
    A = rb.colmajor(torch.from_numpy(a).cuda())
    lu = rb.colmajor(A)
    rb.lu_nopiv_rl(lu, nb=256, outer=outer)
    rng = np.random.default_rng(n)
    b = torch.from_numpy(rng.standard_normal(n)).cuda()
    x_ref, it_ref, be_ref = rb.refine(A, lu, b, tol=1e-14)
    for _ in range(2):
        x = torch.full((n,), float("nan"), dtype=torch.float64, device="cuda")
        it, be = rb.api.refine_static(A, lu, b, x, tol=1e-14)
        torch.cuda.synchronize()
        assert it == it_ref and be == be_ref
        assert torch.equal(x, x_ref)
    assert be_ref <= 1e-14


@pytest.mark.gpu
def test_static_n_zero(built):
    L = _lib.lib()
    it = ctypes.c_int(-1)
    st = L.lu_refine_static_c(None, 0, None, 1, None, 1, None, None, 1e-14, 30,
                              ctypes.byref(it), None)
    assert st == _lib.SUCCESS and it.value == 0
