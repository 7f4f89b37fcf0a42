"""The block-row step of the host entry's left-looking chunk catch-up
(lu_catchup_row_step_c): R -= La Xb (fp16 / bf16 operands, fp32
accumulation), then the unit-lower solve with the step's diagonal block, and
the solved rows' low-precision copy.  The fused one-launch kernel against
the unfused kernels (tensor-core update, blocked U-panel solves) and against
the oracle: with nothing to subtract, the solve is the U part of one outer
step of the reference's right-looking algorithm, bit for bit."""
import ctypes

import numpy as np
import pytest
import torch

import oracle as O
from remifa_b200 import _lib

pytestmark = pytest.mark.gpu


def _st():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def _case(a_host, lda, inn, coff, nc, kl, la, xb, ldx, fused, bf16, part=None):
    """Run one row step on a device copy of a_host (column-major, lda),
    part: optional (ns, nc, ldp) fp32 slabs of partial products; returns
    (matrix, xo) on the host."""
    d = torch.from_numpy(np.asfortranarray(a_host)).cuda()
    d = d.t().contiguous().t() if d.stride(0) != 1 else d
    assert d.stride(0) == 1 and d.stride(1) == lda
    dt = torch.bfloat16 if bf16 else torch.float16
    xo = torch.zeros(nc * ldx, dtype=dt, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    st = _lib.lib().lu_catchup_row_step_c(
        _st(), int(fused), int(bf16), inn, nc, coff, kl, _p(d), lda,
        _p(la) if la is not None else None, la.shape[1] if la is not None else 0,
        _p(xb) if xb is not None else None, _p(xo), ldx,
        _p(part) if part is not None else None,
        part.shape[1] * part.shape[2] if part is not None else 0,
        part.shape[2] if part is not None else 0,
        part.shape[0] if part is not None else 0, _p(err))
    assert st == 0, _lib.lib().lu_last_error()
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    return d.cpu().numpy(), xo


def _block(inn, nc, seed, lda=None, slabs=None):
    """A factored inn x inn diagonal block (the oracle's first outer step of
    a diagonally dominant matrix) and the original block row beside it, in
    one column-major array; plus the oracle's solved block row.  slabs
    (ns x nc x inn, fp32): partial products the step subtracts first; the
    oracle then solves the block row minus their sum (fp32, slab order, one
    subtraction)."""
    n = inn + nc
    a = O.gen_matrix(n, seed=seed, kind=1, alpha=1.5)
    r = np.array(a[:inn, inn:])
    if slabs is not None:
        t = slabs[0, :, :inn].T.copy()
        for sl in slabs[1:]:
            t = t + sl[:, :inn].T            # float32: one rounding per add
        r_eff = r - t                        # one rounding
    else:
        r_eff = r
    f = np.array(a, order="F")
    f[:inn, inn:] = r_eff
    O.lu_rl_steps(f, inn, 0, 0, 1)   # one outer step, FP32 updates
    lda = lda or inn
    m = np.zeros((lda, n), dtype=np.float32, order="F")
    m[:inn, :inn] = f[:inn, :inn]
    m[:inn, inn:] = r
    return m, f[:inn, inn:]


def _operands(inn, nc, kl, ldx, seed, bf16):
    """La (inn x kl, row-major, leading dimension a multiple of 8) and Xb
    (kl x nc, column q at q * ldx), as device tensors, plus their fp64
    values."""
    g = np.random.default_rng(seed)
    dt = torch.bfloat16 if bf16 else torch.float16
    lda_k = (kl + 7) // 8 * 8 + 8
    la64 = g.uniform(-1, 1, (inn, kl)) / np.sqrt(kl)
    xb64 = g.uniform(-1, 1, (kl, nc))
    la = torch.zeros((inn, lda_k), dtype=dt)
    la[:, :kl] = torch.from_numpy(la64)
    xbt = torch.zeros((nc, ldx), dtype=dt)
    xbt[:, :kl] = torch.from_numpy(xb64.T)
    la_v = la[:, :kl].double().numpy()
    xb_v = xbt[:, :kl].double().numpy().T
    return la.cuda(), xbt.reshape(-1).cuda(), la_v, xb_v


@pytest.mark.parametrize("inn,nc,bf16,ns", [(256, 1000, False, 0), (128, 700, True, 0),
                                            (64, 33, False, 0), (256, 32, True, 0),
                                            (256, 1000, False, 3), (128, 97, True, 8)])
def test_row_solve_matches_oracle_bit_for_bit(built, inn, nc, bf16, ns):
    """No product with the previous block row: fused and unfused steps both
    equal the oracle's U part of one outer step exactly -- after the sum of
    ns slabs of partial products is taken off, in the split-K finish's
    order -- and the copy is the solved rows rounded to fp16 / bf16; ragged
    column counts included."""
    slabs = None
    if ns:
        g = np.random.default_rng(ns + nc)
        slabs = (g.uniform(-1, 1, (ns, nc, (inn + 3) // 4 * 4)) * 0.05).astype(np.float32)
    m, want = _block(inn, nc, seed=inn + nc, slabs=slabs)
    part = torch.from_numpy(slabs).cuda() if ns else None
    ldx = inn
    dt = torch.bfloat16 if bf16 else torch.float16
    for fused in (1, 0):
        got, xo = _case(m, inn, inn, inn, nc, 0, None, None, ldx, fused, bf16, part)
        x = got[:inn, inn:inn + nc]
        assert np.array_equal(x, want), (fused, np.abs(x - want).max())
        copy = xo.reshape(nc, ldx)[:, :inn].cpu()
        assert torch.equal(copy, torch.from_numpy(np.ascontiguousarray(x.T)).to(dt))


@pytest.mark.parametrize("inn,nc,kl,bf16,pad", [(256, 4096, 256, False, 0),
                                                (256, 1000, 256, True, 0),
                                                (128, 777, 128, False, 3),
                                                (64, 96, 256, True, 1)])
def test_row_step_with_product(built, inn, nc, kl, bf16, pad):
    """R -= La Xb, then the solve: the fused kernel (mma.sync products) and
    the unfused one (tcgen05 update) agree to fp32 accumulation order, and
    both match the fp64 result; lda not a multiple of 4 (pad) takes the
    4-byte copy paths."""
    lda = inn + pad
    m, _ = _block(inn, nc, seed=3 * inn + nc, lda=lda)
    ldx = max(inn, kl) + 8
    la, xb, la_v, xb_v = _operands(inn, nc, kl, ldx, seed=nc, bf16=bf16)
    outs = [_case(m, lda, inn, inn, nc, kl, la, xb, ldx, fused, bf16)[0]
            for fused in (1, 0)]
    L = np.tril(m[:inn, :inn].astype(np.float64), -1) + np.eye(inn)
    r = m[:inn, inn:inn + nc].astype(np.float64) - la_v @ xb_v
    want = np.linalg.solve(L, r)
    scale = np.abs(want).max()
    xf, xu = (o[:inn, inn:inn + nc] for o in outs)
    # fp32 sums of kl fp16 products (|La Xb| ~ 0.5, sum of |terms| ~ 4)
    assert np.abs(xf - want).max() / scale < 1e-4
    assert np.abs(xu - want).max() / scale < 1e-4
    assert np.abs(xf - xu).max() / scale < 1e-4
    # nothing outside the block row moved
    for o in outs:
        assert np.array_equal(o[:inn, :inn], m[:inn, :inn])


def test_row_step_rejects_unsupported(built):
    """The fused kernel takes multiples of 32 rows up to 256 and K a
    multiple of 32; other shapes are refused, not run."""
    d = torch.zeros((320, 400), dtype=torch.float32, device="cuda")
    xo = torch.zeros(400 * 320, dtype=torch.float16, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    f = _lib.lib().lu_catchup_row_step_c
    for inn, kl in ((288, 0), (48, 0), (64, 40)):
        st = f(_st(), 1, 0, inn, 16, inn, kl, _p(d), 320, _p(xo) if kl else None, 320,
               _p(xo) if kl else None, _p(xo), 320, None, 0, 0, 0, _p(err))
        assert st != 0
