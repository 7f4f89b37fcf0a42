"""GPU tests of the tcgen05 Schur update and the mixed-precision RL path.

The tensor core's internal accumulation order is not specified, so these
tests use stated tolerances: the update must match an fp64 product of the
operands rounded exactly as the oracle rounds them (fp16 / bf16 / e4m3 with
power-of-two tile scales) to within 2 K u32 (|A||B|)_ij."""
import ctypes
import math
import os

import numpy as np
import pytest
import torch

import oracle as O
import remifa_b200 as rb

pytestmark = pytest.mark.gpu
U32 = 2.0 ** -24
REF_SO = os.path.join(os.path.dirname(os.path.dirname(__file__)), "oracle", "_ref",
                      "libremifa_ref.so")


def to_dev(a, lda=None):
    m, n = a.shape
    t = rb.colmajor_empty(m, n, lda if lda is not None else max(m, 1), torch.float32)
    t.copy_(torch.from_numpy(np.ascontiguousarray(a)))
    return t


def to_host(t):
    return np.asfortranarray(t.cpu().numpy())


def pow2_scale(amax, bound=448.0):
    """Largest s with amax * 2^s <= bound (0 for an empty tile)."""
    if not amax > 0:
        return 0
    s = int(math.floor(math.log2(bound / amax)))
    while amax * 2.0 ** (s + 1) <= bound:
        s += 1
    while amax * 2.0 ** s > bound:
        s -= 1
    return s


def split_tiles(X, by_rows):
    """Split fp16 copies of X as the library holds them: per 128-row (A) /
    128-column (B) tile x * 2^s = hi + lo, returned in fp64 with the scale
    divided out again."""
    hi = np.zeros(X.shape)
    lo = np.zeros(X.shape)
    n = X.shape[0] if by_rows else X.shape[1]
    for t in range(0, n, 128):
        blk = X[t:t + 128, :] if by_rows else X[:, t:t + 128]
        s = pow2_scale(float(np.abs(blk).max()), 32768.0)
        xs = (blk.astype(np.float64) * 2.0 ** s).astype(np.float32)
        h = O.round_fmt(xs, O.FMT_FP16)
        l = O.round_fmt((xs - h).astype(np.float32), O.FMT_FP16)
        hv, lv = h.astype(np.float64) * 2.0 ** -s, l.astype(np.float64) * 2.0 ** -s
        if by_rows:
            hi[t:t + 128, :], lo[t:t + 128, :] = hv, lv
        else:
            hi[:, t:t + 128], lo[:, t:t + 128] = hv, lv
    return hi, lo


def rounded_operands(A, B, fmt):
    """The operands exactly as the library's copies hold them, in fp64 and
    with the tile scales divided out again."""
    if fmt != O.FMT_E4M3:
        return (O.round_fmt(A, fmt).astype(np.float64),
                O.round_fmt(B, fmt).astype(np.float64))
    M, K = A.shape
    N = B.shape[1]
    Ar = np.zeros((M, K))
    Br = np.zeros((K, N))
    for t in range(0, M, 128):
        blk = A[t:t + 128, :]
        s = pow2_scale(float(np.abs(blk).max()))
        Ar[t:t + 128, :] = O.round_fmt(blk, fmt, s).astype(np.float64) * 2.0 ** -s
    for t in range(0, N, 128):
        blk = B[:, t:t + 128]
        s = pow2_scale(float(np.abs(blk).max()))
        Br[:, t:t + 128] = O.round_fmt(blk, fmt, s).astype(np.float64) * 2.0 ** -s
    return Ar, Br


KINDS = [(rb.compute_type.TC32, O.FMT_FP16), (rb.compute_type.TC32_BF16, O.FMT_BF16),
         (rb.compute_type.TC32_E4M3, O.FMT_E4M3)]


@pytest.mark.parametrize("compute,fmt", KINDS)
@pytest.mark.parametrize("M,N,K", [(128, 256, 64), (300, 500, 256), (1000, 777, 200),
                                   (2048, 1536, 1024), (5, 7, 3), (96, 40, 16)])
@pytest.mark.parametrize("pad", [0, 3])  # pad 0 (ld % 4 == 0): TMA reduce epilogue
def test_tc_update_matches_rounded_fp64(built, compute, fmt, M, N, K, pad):
    rng = np.random.default_rng(M * 7 + N + K)
    A = np.asfortranarray(rng.standard_normal((M, K)).astype(np.float32))
    B = np.asfortranarray((rng.standard_normal((K, N)) * 3).astype(np.float32))
    C = np.asfortranarray(rng.standard_normal((M, N)).astype(np.float32))
    Ar, Br = rounded_operands(A, B, fmt)
    want = C.astype(np.float64) - Ar @ Br
    bound = 2 * K * U32 * (np.abs(Ar) @ np.abs(Br)) + 2 * U32 * np.abs(want) + 1e-30
    ldc = ((M + 3) // 4) * 4 if pad == 0 else M + 3
    dA, dB, dC = to_dev(A), to_dev(B), to_dev(C, lda=ldc)
    rb.gemmex(compute, -1.0, dA, dB, 1.0, dC)
    torch.cuda.synchronize()
    got = to_host(dC)
    err = np.abs(got - want)
    assert np.all(err <= bound), (err / bound).max()


@pytest.mark.parametrize("M,N,K", [(128, 256, 64), (300, 500, 256), (1000, 777, 200),
                                   (2048, 1536, 1024), (5, 7, 3), (96, 40, 16)])
@pytest.mark.parametrize("pad", [0, 3])
def test_tc_split_update_matches_three_products(built, M, N, K, pad):
    """Split fp16: C - (Ahi Bhi + Ahi Blo + Alo Bhi), fp32 accumulation over
    the 3K concatenated terms; and within ~2^-20 K |A||B| of the fp32-operand
    product, far below the plain fp16 update's 2^-11."""
    rng = np.random.default_rng(M * 5 + N + K)
    A = np.asfortranarray(rng.standard_normal((M, K)).astype(np.float32))
    B = np.asfortranarray((rng.standard_normal((K, N)) * 3).astype(np.float32))
    C = np.asfortranarray(rng.standard_normal((M, N)).astype(np.float32))
    Ah, Al = split_tiles(A, True)
    Bh, Bl = split_tiles(B, False)
    prod = Ah @ Bh + Ah @ Bl + Al @ Bh
    want = C.astype(np.float64) - prod
    mag = np.abs(Ah) @ np.abs(Bh) + np.abs(Ah) @ np.abs(Bl) + np.abs(Al) @ np.abs(Bh)
    bound = 2 * 3 * K * U32 * mag + 2 * U32 * np.abs(want) + 1e-30
    ldc = ((M + 3) // 4) * 4 if pad == 0 else M + 3
    dA, dB, dC = to_dev(A), to_dev(B), to_dev(C, lda=ldc)
    rb.gemmex(rb.compute_type.TC32_SPLIT, -1.0, dA, dB, 1.0, dC)
    torch.cuda.synchronize()
    got = to_host(dC)
    err = np.abs(got - want)
    assert np.all(err <= bound), (err / bound).max()
    exact = C.astype(np.float64) - A.astype(np.float64) @ B.astype(np.float64)
    absab = np.abs(A.astype(np.float64)) @ np.abs(B.astype(np.float64))
    assert np.all(np.abs(got - exact) <= 2.0 ** -20 * K * absab + 4 * U32 * np.abs(exact))


def test_tc_update_repeated_calls_consistent(built):
    # same inputs twice -> same bits (the tile schedule is static)
    rng = np.random.default_rng(0)
    A = np.asfortranarray(rng.standard_normal((1024, 256)).astype(np.float32))
    B = np.asfortranarray(rng.standard_normal((256, 1024)).astype(np.float32))
    outs = []
    for _ in range(2):
        dC = to_dev(np.zeros((1024, 1024), np.float32))
        rb.gemmex(rb.TC32, -1.0, to_dev(A), to_dev(B), 1.0, dC)
        outs.append(to_host(dC))
    torch.cuda.synchronize()
    np.testing.assert_array_equal(outs[0], outs[1])


@pytest.mark.parametrize("m,n,k,compute", [(4096, 4096, 512, rb.TC32),
                                           (3000, 3100, 1000, rb.TC32),
                                           (4352, 4100, 768, rb.compute_type.TC32_BF16)])
def test_pair_update_matches_single_cta(built, m, n, k, compute):
    """A pass of at least 296 tiles of 128 x 256 with K >= 512 runs as CTA
    pairs (tcgen05 cta_group::2, 256 x 256 tiles); the same product cut into 256-column
    slices (too few tiles for pairs) runs on the single-CTA kernel.  Every
    element's sum runs over K in the same order in both, so the results are
    the same bits; they also meet the rounded-operand bound."""
    rng = np.random.default_rng(m + k)
    A = np.asfortranarray(rng.standard_normal((m, k)).astype(np.float32))
    B = np.asfortranarray(rng.standard_normal((k, n)).astype(np.float32))
    C = np.asfortranarray(rng.standard_normal((m, n)).astype(np.float32))
    dA, dB = to_dev(A), to_dev(B)
    whole, sliced = to_dev(C), to_dev(C)
    rb.gemmex(compute, -1.0, dA, dB, 1.0, whole)
    for j in range(0, n, 256):
        rb.gemmex(compute, -1.0, dA, dB[:, j:j + 256], 1.0, sliced[:, j:j + 256])
    torch.cuda.synchronize()
    np.testing.assert_array_equal(to_host(whole), to_host(sliced))
    fmt = O.FMT_FP16 if compute == rb.TC32 else O.FMT_BF16
    Ar = O.round_fmt(A, fmt).astype(np.float64)
    Br = O.round_fmt(B, fmt).astype(np.float64)
    exact = C.astype(np.float64) - Ar @ Br
    err = np.abs(to_host(whole) - exact)
    assert np.all(err <= 2.0 ** -22 * k * (np.abs(Ar) @ np.abs(Br)) + 2 * U32 * np.abs(exact))


@pytest.mark.parametrize("n,nb,compute,fmt", [(512, 128, rb.TC32, O.FMT_FP16),
                                              (1000, 256, rb.TC32, O.FMT_FP16),
                                              (768, 128, rb.compute_type.TC32_BF16, O.FMT_BF16),
                                              (768, 128, rb.compute_type.TC32_E4M3, O.FMT_E4M3),
                                              (768, 128, rb.compute_type.TC32_SPLIT, O.FMT_SPLIT),
                                              (1000, 256, rb.compute_type.TC32_SPLIT, O.FMT_SPLIT)])
def test_lu_rl_mixed_vs_oracle(built, n, nb, compute, fmt):
    a = O.gen_matrix(n, seed=n, kind=1, alpha=1.5)
    want = O.lu_rl(a, nb=nb, outer_fmt=fmt)
    da = to_dev(a)
    info = rb.lu_nopiv_rl(da, nb=nb, outer=compute)
    torch.cuda.synchronize()
    got = to_host(da)
    assert int(info.item()) == 0
    # same algorithm, same rounded operands; only the accumulation order of
    # the tensor core differs from the oracle's fma chain
    rel = np.abs(got - want).max() / np.abs(want).max()
    assert rel < 64 * n * U32, rel
    fe_g, fe_o = O.factor_error(a, got), O.factor_error(a, want)
    assert fe_g <= 2 * fe_o + 1e-7 and fe_o <= 2 * fe_g + 1e-7


@pytest.mark.parametrize("alpha", [1.05, 4.0])
@pytest.mark.parametrize("kscale", [0, 8])
def test_lu_rl_tc32_dominance_and_scale_grid(built, alpha, kscale):
    """The n = 16384 mixed-precision workload's matrix family at a size the
    oracle finishes quickly: row dominance 1.05 / 4 and entries scaled by
    2^0 / 2^8 (fp16 operand range)."""
    n, nb = 1024, 256
    a = O.gen_matrix(n, seed=17, kind=1, alpha=alpha, kscale=kscale)
    want = O.lu_rl(a, nb=nb, outer_fmt=O.FMT_FP16)
    da = to_dev(a)
    info = rb.lu_nopiv_rl(da, nb=nb, outer=rb.TC32)
    torch.cuda.synchronize()
    got = to_host(da)
    assert int(info.item()) == 0
    rel = np.abs(got - want).max() / np.abs(want).max()
    assert rel < 64 * n * U32, rel
    fe_g, fe_o = O.factor_error(a, got), O.factor_error(a, want)
    assert fe_g <= 2 * fe_o + 1e-7 and fe_o <= 2 * fe_g + 1e-7


def test_lu_rl_tc32_vs_reference_gpu(built):
    if not os.path.exists(REF_SO):
        pytest.skip("reference library not built")
    L = ctypes.CDLL(REF_SO)
    vp, i64, i = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int
    L.ref_lu_nopiv_rl_f32.argtypes = [vp, i64, i64, i64, vp, i64, vp, i, i, vp, i64]
    n, nb = 2048, 256
    a = O.gen_diagdom(n, lda=n)
    mine, theirs = to_dev(a), to_dev(a)
    rb.lu_nopiv_rl(mine, nb=nb, outer=rb.TC32)
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    cpy = torch.zeros((n, n), dtype=torch.float16, device="cuda")
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert L.ref_lu_nopiv_rl_f32(st, n, n, nb, ctypes.c_void_p(theirs.data_ptr()), n,
                                 ctypes.c_void_p(info.data_ptr()), 0, 1,
                                 ctypes.c_void_p(cpy.data_ptr()), n) == 0
    torch.cuda.synchronize()
    lm, lr = to_host(mine), to_host(theirs)
    rel = np.abs(lm - lr).max() / np.abs(lr).max()
    assert rel < 1e-3, rel
    x1 = np.ones(n, np.float32)
    b = O.gen_rhs(a, x1)
    e_m = O.nwerr(a, b, O.lu_solve_f32(lm, b))
    e_r = O.nwerr(a, b, O.lu_solve_f32(lr, b))
    c_m = O.cwerr(a, b, O.lu_solve_f32(lm, b), lm)
    c_r = O.cwerr(a, b, O.lu_solve_f32(lr, b), lr)
    assert e_m <= 4 * e_r and e_r <= 4 * e_m, (e_m, e_r)
    assert c_m <= 4 * c_r and c_r <= 4 * c_m, (c_m, c_r)


def test_lu_rl_tc32_large_backward_error(built):
    """n = 8192 through the device generator: size-independent check of the
    solve residual (fp64 on the host) against the FP16-update error level."""
    n = 8192
    da = rb.gen_matrix(n, seed=5, kind=1, alpha=1.5)
    a = to_host(da)
    info = rb.lu_nopiv_rl(da, nb=256, outer=rb.TC32)
    torch.cuda.synchronize()
    assert int(info.item()) == 0
    lu = to_host(da)
    x = O.gen_vector(n, seed=7, kind=1)
    b = np.array(a, np.float64) @ x
    xh = O.lu_solve_f64(lu, b)
    be = O.backward_error(a, b, xh)
    assert be < 1e-4, be


@pytest.mark.parametrize("compute", [rb.FP32, rb.TC32, rb.compute_type.TC32_BF16,
                                     rb.compute_type.TC32_E4M3])
@pytest.mark.parametrize("n,nb", [(1500, 256), (2048, 128), (777, 64)])
def test_lookahead_is_bit_identical(built, compute, n, nb):
    """The look-ahead schedule (panel k+1 concurrent with the bulk update of
    step k on two streams) must not change any element's update order."""
    if compute == rb.compute_type.TC32_E4M3 and nb % 128:
        nb = 128
    a = O.gen_matrix(n, seed=3, kind=1, alpha=1.5)
    d1, d2 = to_dev(a), to_dev(a)
    rb.lu_nopiv_rl(d1, nb=nb, outer=compute, lookahead=False)
    rb.lu_nopiv_rl(d2, nb=nb, outer=compute, lookahead=True, bulk_steps=1)
    torch.cuda.synchronize()
    assert torch.equal(d1, d2)


@pytest.mark.parametrize("compute,fmt", [(rb.TC32, O.FMT_FP16),
                                         (rb.compute_type.TC32_BF16, O.FMT_BF16)])
@pytest.mark.parametrize("n,nb,q", [(2048, 256, 2), (1800, 128, 2), (3000, 256, 2),
                                    (3000, 128, 3), (2500, 128, 4), (4096, 256, 4),
                                    (3000, 256, 0), (3300, 128, 6), (4096, 256, 8),
                                    (2900, 128, 8)])
def test_grouped_bulk_pass(built, compute, fmt, n, nb, q):
    """bulk_steps q (2 .. 8; 0: the default, under look-ahead): q outer
    steps' updates of the bulk of the trailing matrix in one pass,
    C - (L_k U_k + ... + L_k+q-1 U_k+q-1) with one fp32 accumulator, the
    block row and column each step's successors need applied at once with
    every pending product.  Only that rounding differs from the
    step-by-step order: within 64 n u32 of it and of the oracle, same
    ||A - LU|| up to 2x."""
    a = O.gen_matrix(n, seed=n + 11 + q, kind=1, alpha=1.5)
    d1, d2 = to_dev(a), to_dev(a)
    rb.lu_nopiv_rl(d1, nb=nb, outer=compute, bulk_steps=1)
    info = rb.lu_nopiv_rl(d2, nb=nb, outer=compute, bulk_steps=q)
    torch.cuda.synchronize()
    assert int(info.item()) == 0
    one, two = to_host(d1), to_host(d2)
    assert not np.array_equal(one, two)  # the paired passes ran
    want = O.lu_rl(a, nb=nb, outer_fmt=fmt)
    scale = np.abs(want).max()
    assert np.abs(two - one).max() / scale < 64 * n * U32
    assert np.abs(two - want).max() / scale < 64 * n * U32
    fe2, feo = O.factor_error(a, two), O.factor_error(a, want)
    assert fe2 <= 2 * feo + 1e-7 and feo <= 2 * fe2 + 1e-7


@pytest.mark.parametrize("compute", [rb.TC32, rb.TC16, rb.FP16])
@pytest.mark.parametrize("c_half", [False, True])
@pytest.mark.parametrize("M,N,K", [(300, 500, 256), (128, 256, 64), (1000, 777, 200)])
def test_gemmex_fp16_operands(built, compute, c_half, M, N, K):
    """gemmex with fp16 A and B (the reference's TC32 / TC16 / FP16 gemmex
    instantiations): fp32 accumulation of the exact fp16 products, C fp32 or
    rounded to fp16 once."""
    rng = np.random.default_rng(M + N + K)
    A = rng.standard_normal((M, K)).astype(np.float16)
    B = (rng.standard_normal((K, N)) * 3).astype(np.float16)
    C = rng.standard_normal((M, N)).astype(np.float16 if c_half else np.float32)
    want = C.astype(np.float64) - A.astype(np.float64) @ B.astype(np.float64)
    mag = np.abs(A.astype(np.float64)) @ np.abs(B.astype(np.float64))
    bound = 2 * K * U32 * mag + 2 * U32 * np.abs(want) + 1e-30
    if c_half:
        bound = bound + 2.0 ** -11 * np.abs(want) + 2.0 ** -24
    dt = torch.float16
    dA = rb.colmajor(torch.from_numpy(A).cuda(), lda=(M + 7) // 8 * 8)
    dB = rb.colmajor(torch.from_numpy(B).cuda(), lda=(K + 7) // 8 * 8)
    dC = rb.colmajor(torch.from_numpy(C).cuda())
    assert dA.dtype == dt
    rb.gemmex(compute, -1.0, dA, dB, 1.0, dC)
    torch.cuda.synchronize()
    got = np.asfortranarray(dC.double().cpu().numpy())
    err = np.abs(got - want)
    assert np.all(err <= bound), (err / bound).max()


def test_gemmex_fp16_rejections(built):
    a = rb.colmajor_empty(64, 64, 64, torch.float16)
    c = rb.colmajor_empty(64, 64, 64, torch.float32)
    with pytest.raises(NotImplementedError):  # fp16 operands on the SIMT fp32 path
        rb.gemmex(rb.FP32, -1.0, a, a, 1.0, c)
    with pytest.raises(NotImplementedError):  # bf16 kind with fp16 data
        rb.gemmex(rb.compute_type.TC32_BF16, -1.0, a, a, 1.0, c)
