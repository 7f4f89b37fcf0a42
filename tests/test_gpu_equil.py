"""Equilibration on the device (lu_equilibrate_c): LAPACK geequb's power-of-
two row and column scales and laqge's decision, as the reference applies
them on the host before factoring (tests/testing_lu_gpu.hxx:288-311),
checked bit for bit against a host restatement; and its use: a matrix whose
entries lie outside the fp16 range factors with fp16 tensor-core updates
once equilibrated, and refines to an fp64-level backward error."""
import math

import numpy as np
import pytest
import torch

import oracle as O
import remifa_b200 as rb

pytestmark = pytest.mark.gpu
SMLNUM = np.float32(np.finfo(np.float32).tiny)


def _p2(v):
    """2^trunc(log2 v) for v > 0 (trunc toward zero)."""
    m, e = math.frexp(float(v))
    return math.ldexp(1.0, e - 1 if (v >= 1.0 or m == 0.5) else e)


def geequb_laqge(A, force=False):
    n = A.shape[0]
    absA = np.abs(A.astype(np.float64))
    rm = absA.max(axis=1)
    p = np.array([_p2(v) if v > 0 else 0.0 for v in rm])
    rcnd = max(p.min(), SMLNUM) / min(p.max(), 1 / SMLNUM)
    r = (1.0 / np.clip(p, SMLNUM, 1 / SMLNUM)).astype(np.float32)
    cm = (absA * r[:, None].astype(np.float64)).max(axis=0)
    q = np.array([_p2(v) if v > 0 else 0.0 for v in cm])
    ccnd = max(q.min(), SMLNUM) / min(q.max(), 1 / SMLNUM)
    c = (1.0 / np.clip(q, SMLNUM, 1 / SMLNUM)).astype(np.float32)
    amax = absA.max()
    small = float(SMLNUM) / float(np.finfo(np.float32).eps)
    rows = force or rcnd < 0.1 or amax < small or amax > 1 / small
    cols = force or ccnd < 0.1
    equed = ("B" if cols else "R") if rows else ("C" if cols else "N")
    return (r if rows else np.ones(n, np.float32)), (c if cols else np.ones(n, np.float32)), equed


@pytest.mark.parametrize("n,gamma,kscale,force", [(300, 20.0, 0, False), (512, 0.0, 0, False),
                                                  (777, 0.0, 12, True), (1024, 30.0, 3, False)])
def test_equilibrate_matches_geequb_laqge(built, n, gamma, kscale, force):
    a = O.gen_matrix(n, seed=n, kind=1, alpha=1.5, kscale=kscale, gamma_bits=gamma)
    d = rb.colmajor(torch.from_numpy(a).cuda(), lda=n + 1)
    r, c, equed, rowcnd, colcnd, amax = rb.equilibrate(d, force=force)
    torch.cuda.synchronize()
    wr, wc, weq = geequb_laqge(np.array(a), force)
    assert equed == weq
    np.testing.assert_array_equal(r.cpu().numpy(), wr)
    np.testing.assert_array_equal(c.cpu().numpy(), wc)
    scaled = (np.array(a, np.float64) * wr[:, None] * wc[None, :]).astype(np.float32)
    np.testing.assert_array_equal(d.cpu().numpy(), scaled)  # powers of two: exact
    assert amax == float(np.abs(a).max())


def test_equilibration_keeps_fp16_operands_in_range(built):
    """Entries times 2^20 (off-diagonal entries up to ~1e5, beyond fp16's
    65504, in the U12 blocks the tensor cores read): the fp16 trailing update
    overflows without equilibration; with it the factorization is finite and
    refinement reaches 1e-14."""
    n = 1024
    a = rb.gen_matrix(n, seed=4, kind=1, alpha=1.5, kscale=20)
    off = a - torch.diag(torch.diagonal(a))
    assert float(off.abs().max()) > 65504
    g = torch.Generator(device="cuda")
    g.manual_seed(1)
    xt = torch.randn(n, dtype=torch.float64, device="cuda", generator=g)
    b = a.double() @ xt
    lu = rb.colmajor(a)
    info = rb.lu_nopiv_rl(lu, nb=256, outer=rb.TC32)
    torch.cuda.synchronize()
    assert int(info.item()) != 0 or not torch.isfinite(lu).all()
    x, info, it, be = rb.gesv_mixed(a, b, outer=rb.TC32, equilibrate_first=True)
    assert int(info.item()) == 0 and be <= 1e-14, (it, be)
    assert float(((x - xt).abs().max() / xt.abs().max()).item()) < 1e-12
