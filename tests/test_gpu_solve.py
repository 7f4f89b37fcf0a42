"""GPU triangular solves and FP64 iterative refinement, against the FP64
oracle (the reference has no GPU solve; its harness solves on the host)."""
import numpy as np
import pytest
import torch

import oracle as O
import remifa_b200 as rb

pytestmark = pytest.mark.gpu


def to_dev(a, lda=None):
    m, n = a.shape
    t = rb.colmajor_empty(m, n, lda if lda is not None else max(m, 1), torch.float32)
    t.copy_(torch.from_numpy(np.ascontiguousarray(a)))
    return t


def factors(n, seed=1, alpha=1.5, gamma=0.0, outer=rb.FP32):
    a = O.gen_matrix(n, seed=seed, kind=1, alpha=alpha, gamma_bits=gamma)
    da = to_dev(a)
    rb.lu_nopiv_rl(da, nb=256, outer=outer)
    torch.cuda.synchronize()
    return a, da, np.asfortranarray(da.cpu().numpy())


@pytest.mark.parametrize("n", [1, 31, 256, 257, 1000, 2048])
def test_solve_matches_fp64_substitution(built, n):
    a, dlu, lu = factors(n) if n > 1 else (None, None, None)
    if n == 1:
        lu = np.asfortranarray(np.array([[4.0]], np.float32))
        dlu = to_dev(lu)
    rng = np.random.default_rng(n)
    b = rng.standard_normal(n)
    want = O.lu_solve_f64(lu, b)   # fp32 factors, fp64 arithmetic
    x = torch.from_numpy(b.copy()).cuda()
    rb.lu_solve(dlu, x)
    got = x.cpu().numpy()
    assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()


@pytest.mark.parametrize("n,nrhs", [(300, 5), (1100, 64)])
def test_solve_transposed_and_multiple_rhs(built, n, nrhs):
    a, dlu, lu = factors(n, seed=2)
    L = np.tril(lu.astype(np.float64), -1) + np.eye(n)
    U = np.triu(lu.astype(np.float64))
    rng = np.random.default_rng(7)
    B = rng.standard_normal((n, nrhs))
    for trans in (False, True):
        M = (L @ U).T if trans else L @ U
        want = np.linalg.solve(M, B)
        X = torch.from_numpy(np.asfortranarray(B)).cuda().t().contiguous().t()
        rb.lu_solve(dlu, X, trans=trans)
        got = X.cpu().numpy()
        assert np.abs(got - want).max() <= 1e-10 * np.abs(want).max(), trans


@pytest.mark.parametrize("outer,n,gamma", [
    (rb.TC32, 2048, 0.0), (rb.TC32, 4096, 13.0),
    (rb.compute_type.TC32_BF16, 2048, 0.0), (rb.compute_type.TC32_BF16, 4096, 13.0),
    (rb.compute_type.TC32_E4M3, 2048, 0.0), (rb.compute_type.TC32_E4M3, 4096, 4.0),
    (rb.FP32, 4096, 13.0)])
def test_refine_reaches_fp64_backward_error(built, outer, n, gamma):
    """Dominance 1.5 rows scaled by 2^-round(gamma i/(n-1)): kappa ~ 2^gamma.
    (e4m3 factors carry ~2^-4 relative rounding in the trailing updates, so
    classic refinement needs kappa well below 2^4 / update share.)"""
    a = O.gen_matrix(n, seed=11, kind=1, alpha=1.5, gamma_bits=gamma)
    xt = O.gen_vector(n, seed=7, kind=1)
    b = np.array(a, np.float64) @ xt
    da = to_dev(a)
    db = torch.from_numpy(b).cuda()
    x, info, it, be = rb.gesv_mixed(da, db, outer=outer, tol=1e-14)
    torch.cuda.synchronize()
    assert int(info.item()) == 0
    assert be <= 1e-14, (be, it)
    xh = x.cpu().numpy()
    # the oracle's backward error agrees with the device's
    # (the oracle sums sequentially: allow for its own fp64 rounding)
    assert O.backward_error(a, b, xh) < 5e-14
    # forward error bounded by kappa * berr
    assert np.abs(xh - xt).max() / np.abs(xt).max() < 1e-14 * 2.0 ** gamma * 100
    assert it <= 20


def test_refine_reports_non_convergence(built):
    n = 512
    a = O.gen_matrix(n, seed=3, kind=1, alpha=1.5)
    da = to_dev(a)
    lu = rb.colmajor(da)
    rb.lu_nopiv_rl(lu, nb=128, outer=rb.compute_type.TC32_E4M3)
    b = torch.randn(n, dtype=torch.float64, device="cuda")
    # zero iterations allowed: the first solve alone cannot reach 1e-14
    x, it, be = rb.refine(da, lu, b, tol=1e-14, max_iter=0)
    assert it == 0 and be > 1e-14
    with pytest.raises(rb._lib.LuError):
        rb.refine(da, lu, b, tol=1e-14, max_iter=0, raise_on_stall=True)


@pytest.mark.parametrize("n,nrhs,lda_pad,x_off", [
    (64, 1, 0, 0), (65, 3, 1, 1), (127, 9, 3, 0), (500, 17, 1, 1), (1027, 2, 0, 1),
    (2111, 4, 2, 1), (3000, 1, 0, 0)])
def test_solve_layouts_and_groups(built, n, nrhs, lda_pad, x_off):
    """Ragged row blocks, right-hand-side groups of 1/2/4/8 with a partial last
    group, a leading dimension that is not a multiple of 4 (4-byte tile copies)
    and right-hand sides that start off a 16-byte boundary with an odd leading
    dimension (solution blocks read without cp.async)."""
    a, dlu0, lu = factors(n, seed=n)
    dlu = rb.colmajor_empty(n, n, n + lda_pad, torch.float32)
    dlu.copy_(dlu0)
    L = np.tril(lu.astype(np.float64), -1) + np.eye(n)
    U = np.triu(lu.astype(np.float64))
    rng = np.random.default_rng(n + nrhs)
    B = rng.standard_normal((n, nrhs))
    for trans in (False, True):
        M = (L @ U).T if trans else L @ U
        want = np.linalg.solve(M, B)
        buf = rb.colmajor_empty(n + x_off, nrhs, n + x_off + (1 if x_off else 0),
                                torch.float64)
        X = buf[x_off:, :]
        X.copy_(torch.from_numpy(B))
        rb.lu_solve(dlu, X, trans=trans)
        got = X.cpu().numpy()
        assert np.abs(got - want).max() <= 1e-10 * np.abs(want).max(), (trans, n, nrhs)


def test_solve_large_single_rhs(built):
    """n = 8192: 128 row blocks, most of them streaming a backlog of tiles."""
    from scipy.linalg import solve_triangular
    n = 8192
    a = O.gen_matrix(n, seed=5, kind=1, alpha=1.5)
    da = to_dev(a)
    rb.lu_nopiv_rl(da, nb=256, outer=rb.TC32)
    torch.cuda.synchronize()
    lu = np.asfortranarray(da.cpu().numpy())
    f = lu.astype(np.float64)
    rng = np.random.default_rng(3)
    b = rng.standard_normal(n)
    for trans in (False, True):
        if trans:
            want = solve_triangular(f, b, lower=False, trans="T")
            want = solve_triangular(f, want, lower=True, unit_diagonal=True, trans="T")
        else:
            want = O.lu_solve_f64(lu, b)
        x = torch.from_numpy(b.copy()).cuda()
        rb.lu_solve(da, x, trans=trans)
        got = x.cpu().numpy()
        assert np.abs(got - want).max() <= 1e-11 * np.abs(want).max(), trans
