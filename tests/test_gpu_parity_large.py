"""Parity at the sizes the benchmark reports.

n = 16384, nb = 256, fp32 storage with fp16 tensor-core trailing updates
(fp32 accumulation): the default benchmark workload (row dominance 1.5,
entries N(0,1)/sqrt(n), no scaling) and the corners of the dominance x scale
grid (dominance 1.05 / 4, entries scaled by 2^0 / 2^8), each compared with

* the oracle's restatement of the reference algorithm with fp16-rounded
  outer operands (``O.lu_rl(a, 256, outer_fmt=FMT_FP16)``): max relative
  difference < 64 n u32 and ||A - LU||_F / ||A||_F within a factor 2;
* the reference's own ``lu_nopiv_rl<float, FP32, TC32, 8>``
  (src/lu_nopiv.hxx:44-208, cuBLAS inside) on the same device and the same
  matrix: the same relative-difference bound, nwerr and cwerr
  (tests/errors.hxx) within a factor 4.

And the left-looking factorization of an fp16 matrix against the
reference's ``lu_nopiv_ll_f16_tc32xtc32`` (src/lu_nopiv_ll.cxx:282-296) at
the fp16-storage benchmark size (n = 16384, nb = 128) and at n = 2048.

||A - LU||_F is formed in fp64 on the device (a dense fp64 product: the
host would need minutes for n^3 at this size); everything else runs on the
host.  Each case takes about 20 s of oracle time on 16 host cores."""
import ctypes
import os

import numpy as np
import pytest
import torch

import oracle as O
import remifa_b200 as rb

pytestmark = pytest.mark.gpu
U32 = 2.0 ** -24
U16 = 2.0 ** -11
N = 16384
REF_SO = os.path.join(os.path.dirname(os.path.dirname(__file__)), "oracle", "_ref",
                      "libremifa_ref.so")


@pytest.fixture(scope="module")
def ref():
    if not os.path.exists(REF_SO):
        pytest.skip("reference library not built")
    L = ctypes.CDLL(REF_SO)
    vp, i64, i = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int
    L.ref_lu_nopiv_rl_f32.argtypes = [vp, i64, i64, i64, vp, i64, vp, i, i, vp, i64]
    L.ref_lu_nopiv_ll_f16_tc32.argtypes = [vp, i, i, i, vp, i, vp]
    return L


def _st():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def to_host(t: torch.Tensor) -> np.ndarray:
    return np.asfortranarray(t.float().cpu().numpy())


def factor_error_dev(a: torch.Tensor, lu: torch.Tensor) -> float:
    """||A - L U||_F / ||A||_F with L, U taken from the in-place factors `lu`
    (unit lower / upper), all in fp64 on the device."""
    lu64 = lu.double()
    low = torch.tril(lu64, -1)
    low.diagonal().fill_(1.0)
    up = torch.triu(lu64)
    del lu64
    r = a.double() - low @ up
    return float(torch.linalg.norm(r) / torch.linalg.norm(a.double()))


def nw_cw(a: np.ndarray, lu: np.ndarray):
    """The reference's nwerr / cwerr of the fp32 solve with x = 1 (its test
    harness's right-hand side, tests/testing_lu_gpu.hxx:316-351)."""
    b = O.gen_rhs(a, np.ones(a.shape[0], np.float32))
    x = O.lu_solve_f32(lu, b)
    return O.nwerr(a, b, x), O.cwerr(a, b, x, lu)


GRID = [(1.5, 0, 1), (1.05, 0, 2), (1.05, 8, 3), (4.0, 0, 4), (4.0, 8, 5)]


@pytest.mark.parametrize("alpha,kscale,seed", GRID)
def test_tc32_n16384_vs_oracle_and_reference(built, ref, alpha, kscale, seed):
    da = rb.gen_matrix(N, seed=seed, kind=1, alpha=alpha, kscale=kscale)
    a = to_host(da)
    a_dev = da.clone()
    info = rb.lu_nopiv_rl(da, nb=256, outer=rb.TC32)
    theirs = a_dev.clone()
    rinfo = torch.zeros(1, dtype=torch.int32, device="cuda")
    cpy = torch.zeros((N, N), dtype=torch.float16, device="cuda")
    assert ref.ref_lu_nopiv_rl_f32(_st(), N, N, 256, ctypes.c_void_p(theirs.data_ptr()), N,
                                   ctypes.c_void_p(rinfo.data_ptr()), 0, 1,
                                   ctypes.c_void_p(cpy.data_ptr()), N) == 0
    torch.cuda.synchronize()
    del cpy
    assert int(info.item()) == 0
    got, lr = to_host(da), to_host(theirs)
    assert np.isfinite(got).all()

    want = O.lu_rl(a, nb=256, outer_fmt=O.FMT_FP16)
    amax = np.abs(want).max()
    rel_o = np.abs(got - want).max() / amax
    rel_r = np.abs(got - lr).max() / np.abs(lr).max()
    assert rel_o < 64 * N * U32, rel_o
    assert rel_r < 64 * N * U32, rel_r

    fe_g = factor_error_dev(a_dev, da)
    fe_o = factor_error_dev(a_dev, torch.from_numpy(np.ascontiguousarray(want)).cuda())
    fe_r = factor_error_dev(a_dev, theirs)
    assert fe_g <= 2 * fe_o and fe_o <= 2 * fe_g, (fe_g, fe_o)
    assert fe_g <= 4 * fe_r and fe_r <= 4 * fe_g, (fe_g, fe_r)

    nw_g, cw_g = nw_cw(a, got)
    nw_r, cw_r = nw_cw(a, lr)
    assert nw_g <= 4 * nw_r and nw_r <= 4 * nw_g, (nw_g, nw_r)
    assert cw_g <= 4 * cw_r and cw_r <= 4 * cw_g, (cw_g, cw_r)
    print(f"alpha={alpha} k={kscale}: rel vs oracle {rel_o:.2e}, vs reference "
          f"{rel_r:.2e}; ||A-LU||/||A|| mine {fe_g:.2e} oracle {fe_o:.2e} reference "
          f"{fe_r:.2e}; nwerr {nw_g:.2e}/{nw_r:.2e} cwerr {cw_g:.2e}/{cw_r:.2e}")


def _fp16_matrix(n, seed, alpha, kscale=0):
    """An fp16 matrix of the fp16-storage workload's family (on the device)
    and its fp32 copy (exactly the fp16 values)."""
    a32 = rb.gen_matrix(n, seed=seed, kind=1, alpha=alpha, kscale=kscale)
    lda = (n + 7) // 8 * 8
    h = rb.colmajor_empty(n, n, lda, torch.float16)
    rb.convert(a32, h)
    return h, h.float()


@pytest.mark.parametrize("n,nb,alpha,seed", [(2048, 128, 1.5, 21), (2048, 64, 4.0, 22),
                                             (N, 128, 1.5, 1)])
def test_ll_f16_vs_reference(built, ref, n, nb, alpha, seed):
    """fp16 storage, left-looking, fp16 tensor-core updates with fp32
    accumulation.  The reference eliminates the panel in fp16 arithmetic;
    this library eliminates it in fp32 and rounds the results to fp16, so the
    factors differ by a few fp16 units.  Bounds: max relative difference
    < 32 u16 (u16 = 2^-11), nwerr and cwerr of the fp16 factors within a
    factor 4 of the reference's, ||A - LU||_F / ||A||_F no worse than 1.5x."""
    mine, a_dev = _fp16_matrix(n, seed, alpha)
    theirs = mine.clone()
    info = rb.lu_nopiv_ll(mine, nb=nb, outer=rb.TC32)
    rinfo = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert ref.ref_lu_nopiv_ll_f16_tc32(_st(), n, n, nb, ctypes.c_void_p(theirs.data_ptr()),
                                        rb.ld(theirs), ctypes.c_void_p(rinfo.data_ptr())) == 0
    torch.cuda.synchronize()
    assert int(info.item()) == 0
    lm, lr = to_host(mine), to_host(theirs)
    assert np.isfinite(lm).all() and np.isfinite(lr).all()
    rel = np.abs(lm - lr).max() / np.abs(lr).max()
    fe_m = factor_error_dev(a_dev, mine.float())
    fe_r = factor_error_dev(a_dev, theirs.float())
    a = to_host(a_dev)
    nw_m, cw_m = nw_cw(a, lm)
    nw_r, cw_r = nw_cw(a, lr)
    print(f"n={n} nb={nb}: rel {rel:.2e} ({rel / U16:.1f} u16); ||A-LU||/||A|| mine "
          f"{fe_m:.2e} reference {fe_r:.2e}; nwerr {nw_m:.2e}/{nw_r:.2e} cwerr "
          f"{cw_m:.2e}/{cw_r:.2e}")
    assert rel < 32 * U16, rel
    assert fe_m <= 1.5 * fe_r, (fe_m, fe_r)
    assert nw_m <= 4 * nw_r and nw_r <= 4 * nw_m, (nw_m, nw_r)
    assert cw_m <= 4 * cw_r and cw_r <= 4 * cw_m, (cw_m, cw_r)
