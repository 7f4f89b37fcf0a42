"""Left-looking factorization of an fp16 matrix (fp16 storage, fp16
tensor-core updates accumulated in fp32, fp32 panel elimination) against the
oracle's restatement of the same algorithm."""
import numpy as np
import pytest
import torch

import oracle as O
import remifa_b200 as rb

pytestmark = pytest.mark.gpu


def fp16_dev(a, lda):
    m, n = a.shape
    t = rb.colmajor_empty(m, n, lda, torch.float16)
    t.copy_(torch.from_numpy(np.ascontiguousarray(a)).to(torch.float16))
    return t


@pytest.mark.parametrize("n,nb,alpha,k", [(64, 64, 1.5, 0), (300, 64, 1.5, 0),
                                          (1000, 128, 1.5, 0), (1024, 128, 4.0, 0),
                                          (777, 96, 1.05, 0), (2048, 128, 1.5, 8)])
def test_ll_f16_matches_oracle(built, n, nb, alpha, k):
    a = O.round_fmt(O.gen_matrix(n, seed=n + k, kind=1, alpha=alpha, kscale=k), O.FMT_FP16)
    lda = (n + 7) // 8 * 8
    d = fp16_dev(a, lda)
    info = rb.lu_nopiv_ll(d, nb=nb, outer=rb.TC32)
    torch.cuda.synchronize()
    assert int(info.item()) == 0
    got = np.asfortranarray(d.float().cpu().numpy())
    want = O.lu_ll(a, nb=nb, fp16_storage=True)
    # every stored factor is an fp16 number; only the tensor core's
    # accumulation order differs from the oracle's fma chain, which can move
    # an fp16 rounding by one unit
    rel = np.abs(got - want).max() / np.abs(want).max()
    assert rel < 8 * 2.0 ** -11, rel
    fe_g, fe_o = O.factor_error(a, got), O.factor_error(a, want)
    assert fe_g <= 1.5 * fe_o + 1e-6 and fe_o <= 1.5 * fe_g + 1e-6, (fe_g, fe_o)


def test_ll_f16_refines_to_fp64(built):
    """fp16 factors still drive FP64 refinement of the fp32 system."""
    n = 1536
    a = O.round_fmt(O.gen_matrix(n, seed=3, kind=1, alpha=2.0), O.FMT_FP16)
    d = fp16_dev(a, n)
    rb.lu_nopiv_ll(d, nb=128, outer=rb.TC32)
    lu32 = rb.colmajor(d.float())
    A = rb.colmajor(torch.from_numpy(a).cuda())
    b = torch.from_numpy(np.random.default_rng(1).standard_normal(n)).cuda()
    x, it, be = rb.refine(A, lu32, b, tol=1e-14, max_iter=40)
    assert be <= 1e-14, (it, be)


def test_ll_f16_argument_checks(built):
    a = rb.colmajor_empty(100, 100, 100, torch.float16)
    with pytest.raises(ValueError):  # lda not a multiple of 8
        rb.lu_nopiv_ll(a, nb=64, outer=rb.TC32)
    b = rb.colmajor_empty(96, 96, 96, torch.float16)
    with pytest.raises(NotImplementedError):  # fp16 storage needs TC32 updates
        rb.lu_nopiv_ll(b, nb=64, outer=rb.FP32)
    with pytest.raises(NotImplementedError):  # and the left-looking variant
        rb.lu_nopiv_rl(b, nb=64, outer=rb.TC32)


@pytest.mark.parametrize("n,nb", [(1000, 128), (777, 256), (2048, 256)])
def test_ll_f16_panel_fp32_matches_oracle(built, n, nb):
    """OP = OF = fp32 (the reference's ..._fp32xfp32_fp32xfp32 wrappers): the
    block update stays in fp32 until the panel is factored."""
    a = O.round_fmt(O.gen_matrix(n, seed=n + 5, kind=1, alpha=1.5), O.FMT_FP16)
    lda = (n + 7) // 8 * 8
    d = fp16_dev(a, lda)
    info = rb.lu_nopiv_ll(d, nb=nb, outer=rb.TC32, panel_fp32=True)
    torch.cuda.synchronize()
    assert int(info.item()) == 0
    got = np.asfortranarray(d.float().cpu().numpy())
    want = O.lu_ll(a, nb=nb, fp16_storage=True, panel_fp32=True)
    rel = np.abs(got - want).max() / np.abs(want).max()
    assert rel < 8 * 2.0 ** -11, rel
    fe_g, fe_o = O.factor_error(a, got), O.factor_error(a, want)
    assert fe_g <= 1.5 * fe_o + 1e-6 and fe_o <= 1.5 * fe_g + 1e-6, (fe_g, fe_o)


def test_ll_f16_update_kinds(built):
    """fp16 storage: TC16 / FP16 outer and FP16 / TC16 / TC32 inner updates
    (the reference's W = fp16 wrappers) run the same fp32-accumulated tensor
    -core update and fp32 elimination, so they give TC32's factors exactly."""
    n, nb = 640, 128
    a = O.round_fmt(O.gen_matrix(n, seed=9, kind=1, alpha=1.5), O.FMT_FP16)
    base = fp16_dev(a, n)
    rb.lu_nopiv_ll(base, nb=nb, outer=rb.TC32)
    for inner, outer in [(rb.FP16, rb.TC16), (rb.TC16, rb.TC16), (rb.FP16, rb.TC32),
                         (rb.TC32, rb.TC32), (rb.FP16, rb.FP16)]:
        d = fp16_dev(a, n)
        rb.lu_nopiv_ll(d, nb=nb, inner=inner, outer=outer)
        torch.cuda.synchronize()
        assert torch.equal(d, base), (inner, outer)


@pytest.mark.parametrize("panel_fp32", [False, True])
def test_ll_f16_split_k_repeatable(built, panel_fp32):
    """n = 4096, nb = 256: the block-column and block-row updates of the later
    steps are split along K (partial sums in per-split slabs, added in split
    order), so two factorizations of the same matrix give identical factors,
    and they stay within the fp16 tolerance of the oracle's restatement."""
    n, nb = 4096, 256
    a32 = rb.gen_matrix(n, seed=31, kind=1, alpha=1.5)
    src = rb.colmajor_empty(n, n, n, torch.float16)
    rb.convert(a32, src)
    runs = []
    for _ in range(2):
        d = src.clone()
        info = rb.lu_nopiv_ll(d, nb=nb, outer=rb.TC32, panel_fp32=panel_fp32)
        torch.cuda.synchronize()
        assert int(info.item()) == 0
        runs.append(d)
    assert torch.equal(runs[0], runs[1])
    a = np.asfortranarray(src.float().cpu().numpy())
    got = np.asfortranarray(runs[0].float().cpu().numpy())
    want = O.lu_ll(a, nb=nb, fp16_storage=True, panel_fp32=panel_fp32)
    rel = np.abs(got - want).max() / np.abs(want).max()
    assert rel < 8 * 2.0 ** -11, rel
