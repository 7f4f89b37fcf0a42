"""Host-side logic of the batched LU (no GPU needed): the size generator,
the bucket map and the plan's argument checks."""
import ctypes

import numpy as np

import remifa_b200 as rb
from remifa_b200 import _lib
from remifa_b200.batch import BUCKETS, batch_sizes, bucket_of


def test_batch_sizes_log_uniform_and_deterministic():
    s = batch_sizes(10_000, seed=11)
    assert s.dtype == np.int32 and s.shape == (10_000,)
    assert s.min() >= 16 and s.max() <= 511
    assert np.array_equal(s, batch_sizes(10_000, seed=11))
    # log-uniform: each octave [16,32), [32,64), ... holds about a fifth
    counts = np.histogram(np.log2(s), bins=[4, 5, 6, 7, 8, 9])[0]
    assert np.all(np.abs(counts / 10_000 - 0.2) < 0.02), counts
    # about 9e10 flops in total at these sizes
    fl = (2.0 * s.astype(np.float64) ** 3 / 3).sum()
    assert 7e10 < fl < 1.1e11, fl


def test_bucket_map():
    assert [bucket_of(n) for n in (1, 31, 32, 63, 64, 127, 128, 255, 256, 511, 512)] == \
        [0, 0, 1, 1, 2, 2, 3, 3, 4, 4, 5]
    assert BUCKETS == 6


def _create(sizes, outer=rb.TC32, nb=0, tuning=None):
    o = rb.make_opts(nb=nb, outer=outer)
    h = np.ascontiguousarray(sizes, np.int32)
    p = ctypes.c_void_p()
    return _lib.lib().lu_batch_plan_create(ctypes.byref(o), len(h),
                                           h.ctypes.data_as(ctypes.c_void_p),
                                           tuning, ctypes.byref(p))


def test_plan_rejects_bad_arguments_before_touching_the_device():
    assert _create([16, 0, 20]) == _lib.ERR_INVALID_ARG
    assert _create([16, 513]) == _lib.ERR_INVALID_ARG
    assert _create([16], nb=48) == _lib.ERR_INVALID_ARG
    assert _create([16], outer=rb.compute_type.TC32_BF16) == _lib.ERR_UNSUPPORTED
    t = _lib.LuBatchTuning()
    for b in range(BUCKETS):
        t.nb[b], t.outer[b] = 16, int(rb.TC32)
    assert _create([16], tuning=ctypes.byref(t)) == _lib.ERR_INVALID_ARG
