"""lu_panel_c with fp16 storage (remifa::lu_nopiv_panel<half,8>, fp16
arithmetic) bit for bit against the reference's own kernel on the same
device and against the oracle's restatement."""
import ctypes
import os

import numpy as np
import pytest
import torch

import oracle as O
import remifa_b200 as rb
from remifa_b200 import _lib

pytestmark = pytest.mark.gpu
REF_SO = os.path.join(os.path.dirname(os.path.dirname(__file__)), "oracle", "_ref",
                      "libremifa_ref.so")


def _panel(m, seed, scale):
    rng = np.random.default_rng(seed)
    a = rng.standard_normal((m, m)) * scale
    a[np.arange(8), np.arange(8)] += 6.0 * scale
    return np.asfortranarray(a.astype(np.float16))


@pytest.mark.parametrize("m,seed,scale", [(64, 1, 1.0), (200, 2, 30.0), (1000, 3, 0.01),
                                          (8, 4, 1.0)])
def test_panel_f16_bit_exact(built, m, seed, scale):
    a16 = _panel(m, seed, scale)
    d16 = np.asfortranarray(a16[:8, :8].copy())
    dev = lambda x: rb.colmajor(torch.from_numpy(np.ascontiguousarray(x)).cuda())
    mine, d_mine = dev(a16), dev(d16)
    st = torch.zeros(1, dtype=torch.int32, device="cuda")
    rb.lu_nopiv_panel(m, 8, d_mine, mine, mine, st)
    torch.cuda.synchronize()
    got = np.asfortranarray(mine.cpu().numpy())
    want = np.array(a16.astype(np.float32), order="F")
    O.panel_f16(m, 8, np.asfortranarray(a16[:8, :8].astype(np.float32)), want)
    np.testing.assert_array_equal(got.astype(np.float32), want)
    if not os.path.exists(REF_SO):
        pytest.skip("reference library not built")
    L = ctypes.CDLL(REF_SO)
    vp, i = ctypes.c_void_p, ctypes.c_int
    L.ref_panel_f16.argtypes = [vp, i, i, vp, i, vp, i, vp, i, vp]
    theirs, d_theirs = dev(a16), dev(d16)
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert L.ref_panel_f16(s, m, 8, ctypes.c_void_p(d_theirs.data_ptr()), 8,
                           ctypes.c_void_p(theirs.data_ptr()), m,
                           ctypes.c_void_p(theirs.data_ptr()), m,
                           ctypes.c_void_p(st.data_ptr())) == 0
    torch.cuda.synchronize()
    np.testing.assert_array_equal(got, np.asfortranarray(theirs.cpu().numpy()))
