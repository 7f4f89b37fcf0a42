"""The library computes every pivot's 1/d with its own correctly rounded
reciprocal (FMA Newton-Raphson on the hardware approximation); it must equal
CUDA's __frcp_rn for every float input."""
import ctypes

import pytest
import torch

from remifa_b200 import _lib

pytestmark = pytest.mark.gpu


def test_reciprocal_matches_frcp_rn_for_all_floats(built):
    bad = torch.zeros(1, dtype=torch.int64, device="cuda")
    st = _lib.lib().lu_selfcheck_rcp_c(None, ctypes.c_void_p(bad.data_ptr()))
    assert st == _lib.SUCCESS
    torch.cuda.synchronize()
    assert int(bad.item()) == 0
