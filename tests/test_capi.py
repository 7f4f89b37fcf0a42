"""CPU tests of the C ABI boundary: the library loads, exports every symbol
include/lu_b200.h declares, validates arguments before touching a device, and
refuses to run without an sm_100 device (no CPU fallback)."""
import ctypes
import os
import re

import pytest

from remifa_b200 import _lib
import remifa_b200 as rb

HEADER = os.path.join(os.path.dirname(os.path.dirname(__file__)), "include", "lu_b200.h")


def declared_functions():
    src = open(HEADER).read()
    return re.findall(r"LU_API\s+[\w\s\*]+?\b(lu_\w+)\s*\(", src)


def test_library_exports_every_declared_symbol(built):
    names = declared_functions()
    assert len(names) >= 10
    L = _lib.lib()
    for n in names:
        assert hasattr(L, n), n
    # the ctypes table covers the whole header
    assert set(names) <= set(_lib.SIGNATURES), set(names) - set(_lib.SIGNATURES)


def test_opts_default_and_version(built):
    o = _lib.LuOpts()
    _lib.lib().lu_opts_default(ctypes.byref(o))
    assert (o.nb, o.ib, o.inner_update, o.outer_update, o.variant, o.lookahead) == \
        (256, 8, 0, 0, 0, 1)
    assert _lib.lib().lu_abi_version() == 1
    for s in range(9):
        assert _lib.lib().lu_status_string(s)


def _ws(o, m, n, dtype=_lib.F32):
    sz = ctypes.c_size_t(0)
    st = _lib.lib().lu_workspace_size(ctypes.byref(o), m, n, dtype, ctypes.byref(sz))
    return st, sz.value


def test_workspace_size_validation(built):
    o = rb.make_opts()
    st, sz = _ws(o, 1024, 1024)
    assert st == _lib.SUCCESS and sz > 0
    assert _ws(o, 1024, 512)[0] == _lib.ERR_UNSUPPORTED      # square only
    o.nb = 100
    assert _ws(o, 64, 64)[0] == _lib.ERR_INVALID_ARG          # nb % 8 != 0
    o = rb.make_opts()
    o.ib = 4
    assert _ws(o, 64, 64)[0] == _lib.ERR_UNSUPPORTED          # ib is 8
    o = rb.make_opts(diag_width=129)
    assert _ws(o, 64, 64)[0] == _lib.ERR_INVALID_ARG
    # steps per bulk pass: 0 (default) and 1 .. 8; the workspace grows with q
    # (q + 2 operand buffers under look-ahead with fp16 updates)
    sizes = []
    for q in (0, 1, 2, 4, 6, 8):
        st, sz = _ws(rb.make_opts(outer=rb.TC32, bulk_steps=q), 4096, 4096)
        assert st == _lib.SUCCESS, q
        sizes.append(sz)
    assert sizes[0] == sizes[4] and sizes[2] < sizes[3] < sizes[4] < sizes[5]
    for q in (-1, 9):
        assert _ws(rb.make_opts(bulk_steps=q), 64, 64)[0] == _lib.ERR_INVALID_ARG


def _rl(m=64, n=64, a=1, lda=64, info=1, dtype=_lib.F32, ws=None, ws_bytes=0):
    o = rb.make_opts()
    return _lib.lib().lu_nopiv_rl_c(ctypes.byref(o), None, m, n,
                                    ctypes.c_void_p(a) if a else None, dtype, lda,
                                    ctypes.c_void_p(info) if info else None,
                                    None, 0, ws, ws_bytes)


def test_factor_argument_validation_without_device(built):
    # argument errors are reported before any device call
    assert _rl(info=0) == _lib.ERR_INVALID_ARG
    assert _rl(lda=10) == _lib.ERR_INVALID_ARG
    assert _rl(a=0) == _lib.ERR_INVALID_ARG
    assert _rl(m=-1) == _lib.ERR_INVALID_ARG
    assert _rl(ws=ctypes.c_void_p(64), ws_bytes=1) in (_lib.ERR_WORKSPACE,
                                                       _lib.ERR_NO_DEVICE)


def _rl_host(n=64, h=1, lda=64, d=1, ldda=64, info=1, variant=None):
    o = rb.make_opts()
    if variant is not None:
        o.variant = variant
    vp = lambda x: ctypes.c_void_p(x) if x else None
    return _lib.lib().lu_nopiv_rl_host_c(ctypes.byref(o), None, n, vp(h), lda, vp(d), ldda,
                                         vp(info), None, 0)


def test_host_entry_argument_validation_without_device(built):
    # the host-memory entry also reports argument errors before any device call
    assert _rl_host(info=0) == _lib.ERR_INVALID_ARG
    assert _rl_host(lda=10) == _lib.ERR_INVALID_ARG
    assert _rl_host(ldda=10) == _lib.ERR_INVALID_ARG
    assert _rl_host(h=0) == _lib.ERR_INVALID_ARG
    assert _rl_host(d=0) == _lib.ERR_INVALID_ARG
    assert _rl_host(n=-1) == _lib.ERR_INVALID_ARG


def test_catchup_row_step_validation_without_device(built):
    """lu_catchup_row_step_c (one block row of the host entry's chunk
    catch-up) rejects bad arguments, and shapes the fused kernel does not
    take, before any device call."""
    L = _lib.lib()
    ok = ctypes.c_void_p(256)

    def step(fused=1, inn=256, nc=64, coff=256, kl=256, a=ok, lda=256, la=ok, lda_k=264,
             xb=ok, xo=ok, ldx=264, part=None, slab=0, ldp=0, ns=0, err=ok):
        return L.lu_catchup_row_step_c(None, fused, 0, inn, nc, coff, kl, a, lda, la, lda_k,
                                       xb, xo, ldx, part, slab, ldp, ns, err)

    bad = _lib.ERR_INVALID_ARG
    assert step(coff=100) == bad          # the block row overlaps the diagonal block
    assert step(a=None) == bad and step(xo=None) == bad and step(err=None) == bad
    assert step(lda=100) == bad and step(ldx=200) == bad
    assert step(la=None) == bad and step(xb=None) == bad and step(lda_k=100) == bad
    assert step(ns=-1) == bad
    assert step(ns=2) == bad              # slabs without a pointer
    assert step(ns=2, part=ok, ldp=128, slab=128 * 64) == bad     # ldp != in
    assert step(ns=2, part=ok, ldp=256, slab=256 * 63) == bad     # slab too small
    uns = _lib.ERR_UNSUPPORTED
    assert step(inn=288, coff=288, lda=288, ldx=296) == uns       # more than 256 rows
    assert step(inn=48, coff=48, lda=48, ldx=264) == uns          # rows not a multiple of 32
    assert step(kl=40, lda_k=48) == uns                           # K not a multiple of 32
    assert step(fused=0, kl=12, lda_k=16) == uns                  # unfused: K % 8
    import torch
    if not torch.cuda.is_available():
        # valid arguments without a device: no fallback
        assert step() == _lib.ERR_NO_DEVICE


def test_no_cpu_fallback(built):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    # valid arguments, no device: the call must fail, not compute on the host
    assert _rl() == _lib.ERR_NO_DEVICE
    assert _rl_host() == _lib.ERR_NO_DEVICE
    # the entry is right-looking by name: opts.variant is overridden
    assert _rl_host(variant=_lib.LEFT_LOOKING) == _lib.ERR_NO_DEVICE
    st = _lib.lib().lu_convert_c(None, 4, 4, ctypes.c_void_p(1), _lib.F32, 4,
                                 ctypes.c_void_p(1), _lib.F16, 4, 0)
    assert st == _lib.ERR_NO_DEVICE


def test_python_layer_raises_like_reference(built):
    with pytest.raises(ValueError):
        _lib.check(_lib.ERR_INVALID_ARG, "x")
    with pytest.raises(NotImplementedError):
        _lib.check(_lib.ERR_UNSUPPORTED, "x")
    with pytest.raises(RuntimeError):
        _lib.check(_lib.ERR_CUDA, "x")
    assert rb.align_lda(100) == 112 and rb.align_lda(16) == 16
    assert rb.align_lda(100, 2) == 128


def test_refine_python_checks_before_the_call(built):
    """refine / refine_static check dtypes, lengths and devices before the C
    call: the C ABI only sees raw pointers, so a float32 or short x would be
    written out of bounds."""
    import torch
    n = 8
    a = torch.zeros((n, n), dtype=torch.float32).t()
    lu = torch.zeros((n, n), dtype=torch.float32).t()
    b = torch.zeros(n, dtype=torch.float64)
    x = torch.zeros(n, dtype=torch.float64)
    bad = [
        dict(b=b.float()),                                  # b float32
        dict(x=x.float()),                                  # x float32
        dict(x=torch.zeros(n - 1, dtype=torch.float64)),    # x too short
        dict(b=torch.zeros((n, 2), dtype=torch.float64)),   # b not a vector
        dict(lu=torch.zeros((n, n), dtype=torch.float64)),  # lu float64
        dict(a=torch.zeros((n, n + 1), dtype=torch.float32)),  # a not square
        dict(x=torch.zeros(2 * n, dtype=torch.float64)[::2]),  # x not contiguous
        dict(),                                             # host tensors
    ]
    for kw in bad:
        args = dict(a=a, lu=lu, b=b, x=x)
        args.update(kw)
        with pytest.raises(ValueError):
            rb.refine(args["a"], args["lu"], args["b"], args["x"])
        with pytest.raises(ValueError):
            rb.api.refine_static(args["a"], args["lu"], args["b"], args["x"])


def test_refine_static_checks_arguments_before_any_device_call(built):
    """lu_refine_static_c rejects bad arguments exactly as lu_refine_c does,
    before looking up its scratch array (which would touch the device)."""
    L = _lib.lib()
    vp = ctypes.c_void_p
    ok = vp(64)
    # null matrix, lda < n, negative max_iter, negative tol
    assert L.lu_refine_static_c(None, 10, None, 10, ok, 10, ok, ok, 1e-14, 30,
                                None, None) == _lib.ERR_INVALID_ARG
    assert L.lu_refine_static_c(None, 10, ok, 9, ok, 10, ok, ok, 1e-14, 30,
                                None, None) == _lib.ERR_INVALID_ARG
    assert L.lu_refine_static_c(None, 10, ok, 10, ok, 10, ok, ok, 1e-14, -1,
                                None, None) == _lib.ERR_INVALID_ARG
    assert L.lu_refine_static_c(None, 10, ok, 10, ok, 10, ok, ok, -1.0, 30,
                                None, None) == _lib.ERR_INVALID_ARG
    import torch
    if not torch.cuda.is_available():
        # valid arguments without a device: no scratch lookup, no fallback
        assert L.lu_refine_static_c(None, 10, ok, 10, ok, 10, ok, ok, 1e-14, 30,
                                    None, None) == _lib.ERR_NO_DEVICE
