"""GPU parity of the FP32 plain path against the oracle (bit for bit) and the
reference's own compiled kernels (oracle/_ref), all through the C ABI."""
import ctypes
import os

import numpy as np
import pytest
import torch

import oracle as O
import remifa_b200 as rb

pytestmark = pytest.mark.gpu

REF_SO = os.path.join(os.path.dirname(os.path.dirname(__file__)), "oracle", "_ref",
                      "libremifa_ref.so")


def to_dev(a: np.ndarray, lda: int | None = None) -> torch.Tensor:
    m, n = a.shape
    t = rb.colmajor_empty(m, n, lda if lda is not None else O.ld(a), torch.float32)
    t.copy_(torch.from_numpy(np.ascontiguousarray(a)))
    return t


def to_host(t: torch.Tensor) -> np.ndarray:
    return np.asfortranarray(t.cpu().numpy())


@pytest.fixture(scope="module")
def ref():
    if not os.path.exists(REF_SO):
        pytest.skip("reference library not built")
    L = ctypes.CDLL(REF_SO)
    vp, i64, i = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int
    L.ref_panel_f32.argtypes = [vp, i, i, vp, i, vp, i, vp, i, vp]
    L.ref_convert_f32_f16.argtypes = [vp, i, i, vp, i, vp, i]
    L.ref_lu_nopiv_rl_f32.argtypes = [vp, i64, i64, i64, vp, i64, vp, i, i, vp, i64]
    return L


def _st():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


# ------------------------------------------------------------ generator

@pytest.mark.parametrize("n,kind,kscale,gamma", [(1, 0, 0, 0.0), (7, 1, 0, 0.0),
                                                  (64, 0, 8, 0.0), (257, 1, 0, 12.0),
                                                  (300, 1, 8, 20.0)])
def test_gen_matrix_bit_exact(built, n, kind, kscale, gamma):
    lda = n + 3
    g = rb.gen_matrix(n, seed=42, kind=kind, alpha=1.5, kscale=kscale,
                      gamma_bits=gamma, lda=lda)
    torch.cuda.synchronize()
    want = O.gen_matrix(n, seed=42, kind=kind, alpha=1.5, kscale=kscale,
                        gamma_bits=gamma, lda=lda)
    np.testing.assert_array_equal(to_host(g), want)


# ------------------------------------------------------------ convert

@pytest.mark.parametrize("dt,fmt", [(torch.float16, 1), (torch.bfloat16, 2),
                                    (torch.float8_e4m3fn, 3)])
@pytest.mark.parametrize("m,n,lda", [(64, 33, 64), (37, 5, 41), (4096, 3, 4096)])
def test_convert_bit_exact(built, dt, fmt, m, n, lda):
    rng = np.random.default_rng(m + n)
    a = O.colmajor(m, n, lda)
    a[:, :] = (rng.standard_normal((m, n)) * 300).astype(np.float32)
    for s in (0, -3):
        da = to_dev(a)
        out = rb.colmajor_empty(m, n, lda, dt)
        rb.convert(da, out, scale_log2=s)
        got = out.float().cpu().numpy()
        want = O.round_fmt(a, fmt, s)
        if dt == torch.float16:  # overflow -> inf in both
            np.testing.assert_array_equal(got, want)
        else:
            np.testing.assert_array_equal(got, want)


def test_convert_large_bit_exact(built):
    """8192 x 8192 fp32 -> fp16 (256 MB in, larger than L2), scale 2^-2."""
    n = 8192
    rng = np.random.default_rng(8)
    a = np.asfortranarray((rng.standard_normal((n, n)) * 300).astype(np.float32))
    da = to_dev(a)
    out = rb.colmajor_empty(n, n, n, torch.float16)
    rb.convert(da, out, scale_log2=-2)
    got = out.float().cpu().numpy()
    np.testing.assert_array_equal(got, O.round_fmt(a, 1, -2))


def test_convert_f16_matches_reference(built, ref):
    rng = np.random.default_rng(3)
    m, n = 128, 40
    a = np.asfortranarray((rng.standard_normal((m, n)) * 2e4).astype(np.float32))
    da = to_dev(a)
    mine = rb.colmajor_empty(m, n, m, torch.float16)
    rb.convert(da, mine)
    theirs = torch.zeros((n, m), dtype=torch.float16, device="cuda")
    ref.ref_convert_f32_f16(_st(), m, n, ctypes.c_void_p(da.data_ptr()), m,
                            ctypes.c_void_p(theirs.data_ptr()), m)
    torch.cuda.synchronize()
    assert torch.equal(mine.t().contiguous().view(torch.int16),
                       theirs.view(torch.int16))


# ------------------------------------------------------------ panel

@pytest.mark.parametrize("m,n", [(8, 8), (48, 8), (1000, 8), (20, 5), (9, 1)])
def test_panel_bit_exact_vs_oracle(built, m, n):
    a = O.gen_matrix(m, seed=m, kind=0, alpha=2.0, lda=m + 1)
    d = np.asfortranarray(a[:n, :n].copy())
    want = np.array(a, copy=True, order="F")
    O.panel(m, n, d, want)
    da, dd = to_dev(a), to_dev(d)
    stat = torch.zeros(1, dtype=torch.int32, device="cuda")
    rb.lu_nopiv_panel(m, n, dd, da, da, stat)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(to_host(da), want)
    assert int(stat.item()) == n


def test_panel_bit_exact_vs_reference(built, ref):
    m = 520
    a = O.gen_diagdom(m, lda=m)
    d = np.asfortranarray(a[:8, :8].copy())
    mine, theirs, dd = to_dev(a), to_dev(a), to_dev(d)
    rb.lu_nopiv_panel(m, 8, dd, mine, mine)
    stat = torch.zeros(1, dtype=torch.int32, device="cuda")
    ref.ref_panel_f32(_st(), m, 8, ctypes.c_void_p(dd.data_ptr()), 8,
                      ctypes.c_void_p(theirs.data_ptr()), m,
                      ctypes.c_void_p(theirs.data_ptr()), m,
                      ctypes.c_void_p(stat.data_ptr()))
    torch.cuda.synchronize()
    assert torch.equal(mine, theirs)


# ------------------------------------------------------------ gemm

@pytest.mark.parametrize("m,n,k,lda", [(128, 128, 8, 128), (300, 77, 256, 301),
                                       (1, 1, 1, 1), (513, 1029, 64, 516)])
def test_gemmex_fp32_bit_exact(built, m, n, k, lda):
    rng = np.random.default_rng(k)
    A = O.colmajor(m, k, lda); A[:, :] = rng.standard_normal((m, k)).astype(np.float32)
    B = O.colmajor(k, n, max(k, 1)); B[:, :] = rng.standard_normal((k, n)).astype(np.float32)
    C = O.colmajor(m, n, lda); C[:, :] = rng.standard_normal((m, n)).astype(np.float32)
    want = np.array(C, copy=True, order="F")
    O.gemm_sub(A, B, want)
    dA, dB, dC = to_dev(A), to_dev(B), to_dev(C)
    rb.gemmex(rb.FP32, -1.0, dA, dB, 1.0, dC)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(to_host(dC), want)


# ------------------------------------------------------------ factorization

CASES = [(1, 256, 0), (7, 256, 0), (8, 8, 0), (9, 8, 0), (63, 64, 0), (64, 64, 0),
         (65, 64, 0), (200, 256, 0), (257, 256, 0), (520, 256, 0), (520, 64, 8),
         (1024, 256, 64), (1024, 128, 128), (777, 136, 24), (13, 256, 0),
         (150, 256, 0), (1000, 256, 40)]


@pytest.mark.parametrize("n,nb,dw", CASES)
def test_lu_rl_fp32_bit_exact_vs_oracle(built, n, nb, dw):
    a = (O.gen_matrix(n, seed=n + nb, kind=1, alpha=1.5, lda=n + 5) if n > 1
         else np.asfortranarray(np.array([[3.0]], np.float32)))
    want = O.lu_rl(a, nb=nb)
    da = to_dev(a)
    info = rb.lu_nopiv_rl(da, nb=nb, diag_width=dw)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(to_host(da), want)
    assert int(info.item()) == 0


def test_lu_rl_fp32_bit_exact_diagdom_4096(built):
    n = 4096
    a = O.gen_diagdom(n, lda=n)
    want = O.lu_rl(a, nb=256)
    da = to_dev(a)
    rb.lu_nopiv_rl(da, nb=256)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(to_host(da), want)


@pytest.mark.parametrize("n,nb", [(1024, 256), (4096, 256)])
def test_lu_rl_fp32_vs_reference_gpu(built, ref, n, nb):
    """Same input through the reference's own lu_nopiv_rl (cuBLAS) and ours:
    factors within a stated tolerance, errors within a factor of 4."""
    a = O.gen_diagdom(n, lda=n)
    mine, theirs = to_dev(a), to_dev(a)
    rb.lu_nopiv_rl(mine, nb=nb)
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = ref.ref_lu_nopiv_rl_f32(_st(), n, n, nb, ctypes.c_void_p(theirs.data_ptr()),
                                 n, ctypes.c_void_p(info.data_ptr()), 0, 0, None, 0)
    assert rc == 0
    torch.cuda.synchronize()
    lm, lr = to_host(mine), to_host(theirs)
    U32 = 2.0 ** -24
    rel = np.abs(lm - lr).max() / np.abs(lr).max()
    assert rel <= 4 * n * U32, rel
    x1 = np.ones(n, np.float32)
    b = O.gen_rhs(a, x1)
    e_m = O.nwerr(a, b, O.lu_solve_f32(lm, b))
    e_r = O.nwerr(a, b, O.lu_solve_f32(lr, b))
    assert e_m <= 4 * e_r and e_r <= 4 * e_m, (e_m, e_r)


def test_zero_pivot_reported(built):
    n = 64
    a = O.gen_matrix(n, seed=1, kind=0, alpha=2.0)
    a[:, 20] = 0.0
    a[20, :] = 0.0  # column 20 of the factor is exactly zero -> pivot 21
    da = to_dev(a)
    info = rb.lu_nopiv_rl(da, nb=32)
    torch.cuda.synchronize()
    assert int(info.item()) == 21


def test_lowp_copy_side_effect(built):
    n = 100
    a = O.gen_matrix(n, seed=4, kind=0, alpha=2.0)
    da = to_dev(a)
    cpy = rb.colmajor_empty(n, n, 104, torch.float16)
    rb.lu_nopiv_rl(da, nb=64, a_cpy=cpy)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(cpy.float().cpu().numpy(),
                                  O.round_fmt(to_host(da), 1))


def test_workspace_caller_provided(built):
    n = 300
    a = O.gen_matrix(n, seed=8, kind=1, alpha=2.0)
    ws = torch.empty(rb.workspace_size(n), dtype=torch.uint8, device="cuda")
    da = to_dev(a)
    rb.lu_nopiv_rl(da, nb=128, workspace=ws)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(to_host(da), O.lu_rl(a, nb=128))
    with pytest.raises(RuntimeError):
        rb.lu_nopiv_rl(to_dev(a), nb=128, workspace=ws[:1])


# ------------------------------------------------------------ left-looking

# nb > 128: outer blocks factored as 128-wide sub-blocks (the oracle restates
# that nesting with sub = 128)
LL_CASES = [(7, 8), (64, 64), (200, 64), (257, 128), (520, 64), (1024, 128), (777, 32),
            (1000, 256), (777, 192), (300, 512)]


@pytest.mark.parametrize("n,nb", LL_CASES)
def test_lu_ll_fp32_bit_exact_vs_oracle(built, n, nb):
    a = O.gen_matrix(n, seed=n + 3, kind=1, alpha=1.5, lda=n + 2)
    want = O.lu_ll(a, nb=nb)
    da = to_dev(a)
    info = rb.lu_nopiv_ll(da, nb=nb)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(to_host(da), want)
    assert int(info.item()) == 0


def test_lu_ll_fp32_vs_reference_gpu(built):
    if not os.path.exists(REF_SO):
        pytest.skip("reference library not built")
    L = ctypes.CDLL(REF_SO)
    vp, i = ctypes.c_void_p, ctypes.c_int
    L.ref_lu_nopiv_ll_f32.argtypes = [vp, i, i, i, vp, i, vp]
    n, nb = 1024, 64
    a = O.gen_diagdom(n, lda=n)
    mine, theirs = to_dev(a), to_dev(a)
    rb.lu_nopiv_ll(mine, nb=nb)
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert L.ref_lu_nopiv_ll_f32(_st(), n, n, nb, ctypes.c_void_p(theirs.data_ptr()), n,
                                 ctypes.c_void_p(info.data_ptr())) == 0
    torch.cuda.synchronize()
    lm, lr = to_host(mine), to_host(theirs)
    assert np.abs(lm - lr).max() / np.abs(lr).max() <= 4 * n * 2.0 ** -24
    b = O.gen_rhs(a, np.ones(n, np.float32))
    e_m = O.nwerr(a, b, O.lu_solve_f32(lm, b))
    e_r = O.nwerr(a, b, O.lu_solve_f32(lr, b))
    assert e_m <= 4 * e_r and e_r <= 4 * e_m


def test_lu_ll_tensor_core_split_k_repeatable(built):
    """n = 4096, nb = 256 on fp32 storage: the later steps' K = ofs updates
    run split along K; the partial sums are added in a fixed order, so the
    factors are identical run to run."""
    n, nb = 4096, 256
    a = rb.gen_matrix(n, seed=32, kind=1, alpha=1.5)
    runs = []
    for _ in range(2):
        d = rb.colmajor(a.clone())
        info = rb.lu_nopiv_ll(d, nb=nb, outer=rb.TC32)
        torch.cuda.synchronize()
        assert int(info.item()) == 0
        runs.append(d)
    assert torch.equal(runs[0], runs[1])
    fe = O.factor_error(to_host(a), to_host(runs[0]))
    assert fe < 2e-4, fe


@pytest.mark.parametrize("compute", [rb.TC32, rb.compute_type.TC32_BF16])
def test_lu_ll_tensor_core(built, compute):
    n, nb = 1500, 128
    a = O.gen_matrix(n, seed=5, kind=1, alpha=1.5)
    da = to_dev(a)
    info = rb.lu_nopiv_ll(da, nb=nb, outer=compute)
    torch.cuda.synchronize()
    assert int(info.item()) == 0
    got = to_host(da)
    fe = O.factor_error(a, got)
    assert fe < (2e-4 if compute == rb.TC32 else 2e-3), fe
    # same algorithm in fp32: close to the FP32 Crout factors
    want = O.lu_ll(a, nb=nb)
    assert np.abs(got - want).max() / np.abs(want).max() < (1e-3 if compute == rb.TC32 else 1e-2)


def test_lu_ll_limits(built):
    a = to_dev(O.gen_matrix(300, seed=1, kind=0, alpha=2.0))
    with pytest.raises(NotImplementedError):
        rb.lu_nopiv_ll(a, nb=128, outer=rb.compute_type.TC32_E4M3)
    with pytest.raises(NotImplementedError):  # fp16 inner updates need fp16 storage
        rb.lu_nopiv_ll(a, nb=128, inner=rb.FP16)


def test_lu_ll_nb256_vs_reference_gpu(built):
    """The reference's default outer block (nb = 256) on the left-looking
    variant: the reference factors it with one 8-column Crout loop, this
    library as two 128-wide sub-blocks; same factors up to rounding."""
    if not os.path.exists(REF_SO):
        pytest.skip("reference library not built")
    L = ctypes.CDLL(REF_SO)
    vp, i = ctypes.c_void_p, ctypes.c_int
    L.ref_lu_nopiv_ll_f32.argtypes = [vp, i, i, i, vp, i, vp]
    n, nb = 1024, 256
    a = O.gen_diagdom(n, lda=n)
    mine, theirs = to_dev(a), to_dev(a)
    rb.lu_nopiv_ll(mine, nb=nb)
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert L.ref_lu_nopiv_ll_f32(_st(), n, n, nb, ctypes.c_void_p(theirs.data_ptr()), n,
                                 ctypes.c_void_p(info.data_ptr())) == 0
    torch.cuda.synchronize()
    lm, lr = to_host(mine), to_host(theirs)
    assert np.abs(lm - lr).max() / np.abs(lr).max() <= 4 * n * 2.0 ** -24
    b = O.gen_rhs(a, np.ones(n, np.float32))
    e_m = O.nwerr(a, b, O.lu_solve_f32(lm, b))
    e_r = O.nwerr(a, b, O.lu_solve_f32(lr, b))
    assert e_m <= 4 * e_r and e_r <= 4 * e_m


@pytest.mark.parametrize("n,nb,outer,la,pad", [
    (300, 256, rb.FP32, True, 0),                          # too small to chunk
    (2048, 256, rb.FP32, True, 0),                         # 8 chunks of one block
    (2048, 256, rb.TC32, True, 0),
    (2048, 256, rb.TC32, False, 0),                        # no look-ahead
    (2600, 256, rb.FP32, True, 3),                         # ragged last block, padded lda
    (4000, 256, rb.TC32, True, 0),                         # 2-block chunks, ragged end
    (3000, 128, rb.compute_type.TC32_BF16, True, 1),
    (4096, 256, rb.compute_type.TC32_E4M3, True, 0),       # tile scales per chunk range
    (4096, 256, rb.compute_type.TC32_SPLIT, True, 0),
    (8192, 256, rb.TC32, True, 0)])                        # 4-block chunks: deep steps inside
def test_host_entry_matches_device_entry(built, n, nb, outer, la, pad):
    """lu_nopiv_rl_host_c (host matrix in by column chunks, each chunk caught
    up with the earlier steps, factored and sent back while later chunks
    compute) gives exactly the device entry point's factors."""
    a = O.gen_matrix(n, seed=n + 3, kind=1, alpha=1.5)
    d = rb.colmajor(torch.from_numpy(a).cuda(), lda=n + pad)
    # the host entry applies the outer steps one by one (no two-step bulk pass)
    rb.lu_nopiv_rl(d, nb=nb, outer=outer, lookahead=la, bulk_steps=1)
    h = torch.empty((n, n + pad), dtype=torch.float32, pin_memory=True).t()[:n, :]
    h.copy_(torch.from_numpy(a))
    work = rb.colmajor_empty(n, n, n + 2 * pad, torch.float32)
    info = rb.lu_nopiv_rl_host(h, work, nb=nb, outer=outer, lookahead=la, bulk_steps=1)
    torch.cuda.synchronize()
    assert int(info.item()) == 0
    assert np.array_equal(h.numpy(), d.cpu().numpy())


@pytest.mark.parametrize("n,nb,outer", [(4096, 256, rb.TC32), (3000, 128, rb.compute_type.TC32_BF16),
                                        (8192, 256, rb.TC32), (5000, 256, rb.TC32),
                                        (6144, 128, rb.compute_type.TC32_BF16)])
def test_host_entry_two_step_bulk(built, n, nb, outer):
    """The host entry with several steps per bulk pass (the default): the
    chunk factorizations group their bulk passes and arriving chunks are
    caught up in left-looking order (block-row updates over all earlier
    steps, then the row's solves); same factors as the oracle's
    step-by-step restatement up to those roundings, ragged last chunks and
    blocks included."""
    fmt = O.FMT_FP16 if outer == rb.TC32 else O.FMT_BF16
    a = O.gen_matrix(n, seed=n + 7, kind=1, alpha=1.5)
    h = torch.empty((n, n), dtype=torch.float32, pin_memory=True).t()[:n, :]
    h.copy_(torch.from_numpy(a))
    work = rb.colmajor_empty(n, n, n, torch.float32)
    info = rb.lu_nopiv_rl_host(h, work, nb=nb, outer=outer)
    torch.cuda.synchronize()
    assert int(info.item()) == 0
    got = h.numpy()
    want = O.lu_rl(a, nb=nb, outer_fmt=fmt)
    assert np.abs(got - want).max() / np.abs(want).max() < 64 * n * 2.0 ** -24
    b = O.gen_rhs(a, np.ones(n, np.float32))
    e_g = O.nwerr(a, b, O.lu_solve_f32(np.asfortranarray(got), b))
    e_o = O.nwerr(a, b, O.lu_solve_f32(want, b))
    assert e_g <= 2 * e_o and e_o <= 2 * e_g, (e_g, e_o)


def test_library_pool_reuse_and_trim(built):
    """Without a caller workspace the factorization allocates from the
    library's stream-ordered pool, which keeps the memory between calls;
    lu_trim_memory_c hands it back.  Results are the same either way."""
    n = 2048
    a = rb.gen_matrix(n, seed=41, kind=1, alpha=1.5)
    outs = []
    for trim in (False, False, True):
        d = rb.colmajor(a.clone())
        info = rb.lu_nopiv_rl(d, nb=256, outer=rb.TC32)
        torch.cuda.synchronize()
        assert int(info.item()) == 0
        outs.append(d)
        if trim:
            rb.trim_memory()
    assert torch.equal(outs[0], outs[1]) and torch.equal(outs[1], outs[2])


def test_concurrent_calls_from_two_threads(built):
    """Two host threads factor different matrices at once, each on its own
    stream (the library's internal streams are shared per device; a call is
    enqueued whole under a per-device lock): each result equals the same
    factorization run alone."""
    import threading
    n = 2048
    mats = [rb.gen_matrix(n, seed=50 + i, kind=1, alpha=1.5) for i in range(2)]
    alone = []
    for m in mats:
        d = rb.colmajor(m.clone())
        rb.lu_nopiv_rl(d, nb=256, outer=rb.TC32)
        alone.append(d)
    torch.cuda.synchronize()
    for variant in ("rl", "ll"):
        outs = [rb.colmajor(m.clone()) for m in mats]
        refs = []
        for m in mats:
            d = rb.colmajor(m.clone())
            if variant == "rl":
                rb.lu_nopiv_rl(d, nb=256, outer=rb.TC32)
            else:
                rb.lu_nopiv_ll(d, nb=256, outer=rb.TC32)
            refs.append(d)
        torch.cuda.synchronize()
        streams = [torch.cuda.Stream() for _ in mats]
        errs = []

        def work(i):
            try:
                for _ in range(3):
                    with torch.cuda.stream(streams[i]):
                        outs[i].copy_(mats[i])
                        if variant == "rl":
                            rb.lu_nopiv_rl(outs[i], nb=256, outer=rb.TC32, stream=streams[i])
                        else:
                            rb.lu_nopiv_ll(outs[i], nb=256, outer=rb.TC32, stream=streams[i])
                    streams[i].synchronize()
            except Exception as e:  # pragma: no cover - reported below
                errs.append(e)

        ts = [threading.Thread(target=work, args=(i,)) for i in range(2)]
        for t in ts:
            t.start()
        for t in ts:
            t.join()
        torch.cuda.synchronize()
        assert not errs, errs
        for i in range(2):
            assert torch.equal(outs[i], refs[i]), (variant, i)
