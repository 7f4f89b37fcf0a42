"""Differentiable solve (lu_adjoint_c behind torch.autograd): gradients
against dense FP64 formulas and a central finite difference.  The reference
has no derivative of its LU, so the checker is the calculus itself:
dL/dB = A^-T G, dL/dA = -(A^-T G) X^T."""
import numpy as np
import pytest
import torch

import oracle as O
import remifa_b200 as rb
from remifa_b200.autograd import lu_solve_autograd

pytestmark = pytest.mark.gpu


def grid_matrix(n, seed, step_bits=12):
    """Diagonally dominant matrix whose entries are multiples of 2^-step_bits
    in [-4, 4] + n on the diagonal: exact in fp32, and A +- h E stays exact
    for h = 2^-10 and integer E."""
    rng = np.random.default_rng(seed)
    q = rng.integers(-4 << step_bits, 4 << step_bits, size=(n, n))
    a = q.astype(np.float64) / (1 << step_bits)
    a[np.diag_indices(n)] += n
    return a.astype(np.float32)


def dense_grads(a, b, w):
    A = a.astype(np.float64)
    X = np.linalg.solve(A, b)
    dB = np.linalg.solve(A.T, w)
    dA = -dB @ X.T
    return X, dA, dB


@pytest.mark.parametrize("outer,refine", [(rb.FP32, True), (rb.TC32, True),
                                          (rb.FP32, False)])
@pytest.mark.parametrize("n,nrhs", [(64, 1), (200, 3), (1000, 8)])
def test_gradients_match_dense_fp64(built, outer, refine, n, nrhs):
    a = grid_matrix(n, seed=n + nrhs)
    rng = np.random.default_rng(3)
    b = rng.standard_normal((n, nrhs))
    w = rng.standard_normal((n, nrhs))
    X_ref, dA_ref, dB_ref = dense_grads(a, b, w)
    A = torch.from_numpy(a).cuda().requires_grad_(True)
    B = torch.from_numpy(b).cuda().requires_grad_(True)
    X = lu_solve_autograd(A, B, outer=outer, nb=128, refine=refine)
    (X * torch.from_numpy(w).cuda()).sum().backward()
    tol = 1e-13 if refine else 1e-5
    x = X.detach().cpu().numpy()
    assert np.abs(x - X_ref).max() <= tol * np.abs(X_ref).max() * 10
    db = B.grad.cpu().numpy()
    assert np.abs(db - dB_ref).max() <= tol * np.abs(dB_ref).max() * 10
    da = A.grad.cpu().numpy().astype(np.float64)
    # dA is stored fp32: half an ulp of rounding on top of the solve error
    assert np.abs(da - dA_ref).max() <= (tol * 10 + 2**-23) * np.abs(dA_ref).max()


def test_vector_rhs_and_b_only(built):
    n = 96
    a = grid_matrix(n, seed=5)
    b = np.random.default_rng(1).standard_normal(n)
    A = torch.from_numpy(a).cuda()
    B = torch.from_numpy(b).cuda().requires_grad_(True)
    X = lu_solve_autograd(A, B, outer=rb.FP32, nb=64)
    assert X.shape == (n,)
    X.sum().backward()
    want = np.linalg.solve(a.astype(np.float64).T, np.ones(n))
    assert np.abs(B.grad.cpu().numpy() - want).max() <= 1e-13 * np.abs(want).max()
    assert A.grad is None


def test_finite_difference_n64(built):
    """Central difference of L(A) = w . A^-1 b along an integer direction E,
    with A +- hE exact in fp32 and every solve refined to fp64 level."""
    n = 64
    a = grid_matrix(n, seed=11)
    rng = np.random.default_rng(4)
    b = rng.standard_normal(n)
    w = rng.standard_normal(n)
    E = rng.integers(-3, 4, size=(n, n)).astype(np.float32)
    h = 2.0**-10
    Wt = torch.from_numpy(w).cuda()

    def loss(mat):
        Am = torch.from_numpy(mat).cuda()
        return float((lu_solve_autograd(Am, torch.from_numpy(b).cuda(),
                                        outer=rb.FP32, nb=32) * Wt).sum())

    ap, am = a + np.float32(h) * E, a - np.float32(h) * E
    assert np.array_equal(ap.astype(np.float64), a.astype(np.float64) + h * E)
    fd = (loss(ap) - loss(am)) / (2 * h)
    A = torch.from_numpy(a).cuda().requires_grad_(True)
    (lu_solve_autograd(A, torch.from_numpy(b).cuda(), outer=rb.TC32, nb=32)
     * Wt).sum().backward()
    an = float((A.grad.double().cpu() * torch.from_numpy(E).double()).sum())
    assert abs(fd - an) <= 1e-5 * max(abs(an), 1e-3), (fd, an)


def test_adjoint_c_unrefined_matches_oracle_solve(built):
    """lu_adjoint_c without refinement = two transposed substitutions with
    the fp32 factors in fp64 arithmetic (the oracle's solve on A^T)."""
    n, k = 300, 2
    a = O.gen_matrix(n, seed=9, kind=1, alpha=1.5)
    lu = rb.colmajor(torch.from_numpy(a).cuda())
    rb.lu_nopiv_rl(lu, nb=128)
    rng = np.random.default_rng(2)
    g = rng.standard_normal((n, k))
    x = rng.standard_normal((n, k))
    G = torch.from_numpy(np.asfortranarray(g)).cuda().t().contiguous().t()
    Xd = torch.from_numpy(np.asfortranarray(x)).cuda().t().contiguous().t()
    dA = rb.colmajor_empty(n, n, n, torch.float32)
    from remifa_b200.autograd import adjoint
    adjoint(lu, Xd, G, da=dA)
    f = np.asfortranarray(lu.cpu().numpy()).astype(np.float64)
    L = np.tril(f, -1) + np.eye(n)
    U = np.triu(f)
    want = np.linalg.solve((L @ U).T, g)
    got = G.cpu().numpy()
    assert np.abs(got - want).max() <= 1e-10 * np.abs(want).max()
    wantA = (-(got @ x.T)).astype(np.float32)
    assert np.array_equal(dA.cpu().numpy(), wantA) or \
        np.abs(dA.cpu().numpy() - wantA).max() <= 2**-22 * np.abs(wantA).max()


def test_singular_forward_raises(built):
    a = np.eye(8, dtype=np.float32)
    a[3, 3] = 0.0
    with pytest.raises(RuntimeError):
        lu_solve_autograd(torch.from_numpy(a).cuda(), torch.ones(8, dtype=torch.float64,
                                                                   device="cuda"))
