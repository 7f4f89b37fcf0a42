"""Batched solves, FP64 refinement and the batched adjoint (backward of
X_i = A_i^-1 B_i), against dense FP64 formulas per matrix and a central
finite difference."""
import numpy as np
import pytest
import torch

import oracle as O
import remifa_b200 as rb
from remifa_b200.batch import (BatchPlan, MatrixBatch, RhsBatch, batched_lu_solve)

pytestmark = pytest.mark.gpu


def host_a(mats, i):
    return np.asfortranarray(mats.matrix(i).cpu().numpy())


def make(sizes, seed, outer=rb.TC32, nrhs=1):
    a = MatrixBatch(sizes, align=4).generate(seed=seed)
    lu = a.like(a.data.clone())
    plan = BatchPlan(sizes, outer=outer)
    info = plan(lu)
    torch.cuda.synchronize()
    assert int(info.abs().sum()) == 0
    rng = np.random.default_rng(seed)
    b = RhsBatch(sizes, nrhs)
    b.data.copy_(torch.from_numpy(rng.standard_normal(b.data.numel())))
    return a, lu, plan, b


@pytest.mark.parametrize("trans", [False, True])
def test_batch_solve_matches_fp64_substitution(built, trans):
    sizes = np.array([2, 7, 33, 64, 100, 255, 256, 300, 512], np.int32)
    a, lu, plan, b = make(sizes, 3, outer=rb.FP32, nrhs=2)
    x = b.like(b.data.clone())
    plan.solve(lu, x, trans=trans)
    torch.cuda.synchronize()
    for i, n in enumerate(sizes):
        f = host_a(lu, i).astype(np.float64)
        L = np.tril(f, -1) + np.eye(n)
        U = np.triu(f)
        M = (L @ U).T if trans else L @ U
        want = np.linalg.solve(M, b.block(i).cpu().numpy())
        got = x.block(i).cpu().numpy()
        assert np.abs(got - want).max() <= 1e-11 * max(np.abs(want).max(), 1e-300), n


@pytest.mark.parametrize("trans", [False, True])
def test_batch_refinement_reaches_fp64_backward_error(built, trans):
    rng = np.random.default_rng(5)
    sizes = rng.integers(64, 257, size=200).astype(np.int32)
    a, lu, plan, b = make(sizes, 7, outer=rb.TC32, nrhs=3)
    x = b.like(b.data.clone())
    plan.solve(lu, x, a=a, trans=trans, refine_iters=5)
    torch.cuda.synchronize()
    worst = 0.0
    for i in range(0, len(sizes), 7):
        A = host_a(a, i).astype(np.float64)
        Aop = A.T if trans else A
        X, B = x.block(i).cpu().numpy(), b.block(i).cpu().numpy()
        r = B - Aop @ X
        be = np.abs(r).max() / (np.abs(Aop).sum(axis=1).max() * np.abs(X).max() +
                                np.abs(B).max())
        worst = max(worst, be)
    assert worst <= 1e-14, worst


def test_batch_adjoint_matches_dense_gradients(built):
    rng = np.random.default_rng(9)
    sizes = rng.integers(64, 257, size=64).astype(np.int32)
    a, lu, plan, b = make(sizes, 11, outer=rb.TC32, nrhs=2)
    x = b.like(b.data.clone())
    plan.solve(lu, x, a=a, refine_iters=4)
    g = b.like(torch.from_numpy(rng.standard_normal(b.data.numel())).cuda())
    g0 = g.data.clone()
    da = a.like()
    plan.adjoint(lu, x, g, da=da, a=a, refine_iters=4)
    torch.cuda.synchronize()
    for i in range(0, len(sizes), 5):
        A = host_a(a, i).astype(np.float64)
        X = np.linalg.solve(A, b.block(i).cpu().numpy())
        G = g0[b.offsets[i]:b.offsets[i + 1]].view(2, -1).t().cpu().numpy()
        dB = np.linalg.solve(A.T, G)
        dA = -dB @ X.T
        assert np.abs(g.block(i).cpu().numpy() - dB).max() <= 1e-12 * np.abs(dB).max()
        got = np.asfortranarray(da.matrix(i).cpu().numpy()).astype(np.float64)
        assert np.abs(got - dA).max() <= (1e-12 + 2.0 ** -23) * np.abs(dA).max()


def test_batched_autograd_1024_matrices(built):
    """The batched-backward workload: 1,024 matrices, sizes uniform in
    [64, 256], fp16 tensor-core factors, loss sum(W * X); gradients checked
    against dense FP64 on a sample."""
    rng = np.random.default_rng(12)
    sizes = rng.integers(64, 257, size=1024).astype(np.int32)
    layout = MatrixBatch(sizes, align=4).generate(seed=12, alpha=2.0)
    plan = BatchPlan(sizes, outer=rb.TC32)
    a_flat = layout.data.clone().requires_grad_(True)
    rhs = RhsBatch(sizes, 1)
    b_flat = torch.from_numpy(rng.standard_normal(rhs.data.numel())).cuda().requires_grad_(True)
    w = torch.from_numpy(rng.standard_normal(rhs.data.numel())).cuda()
    x = batched_lu_solve(a_flat, b_flat, layout, plan, nrhs=1, refine_iters=4)
    (x * w).sum().backward()
    torch.cuda.synchronize()
    ga = layout.like(a_flat.grad)
    for i in range(0, 1024, 61):
        n = int(sizes[i])
        A = np.asfortranarray(layout.matrix(i).cpu().numpy()).astype(np.float64)
        o0, o1 = rhs.offsets[i], rhs.offsets[i + 1]
        B = b_flat.detach()[o0:o1].cpu().numpy()
        W = w[o0:o1].cpu().numpy()
        X = np.linalg.solve(A, B)
        dB = np.linalg.solve(A.T, W)
        dA = -np.outer(dB, X)
        assert np.abs(x.detach()[o0:o1].cpu().numpy() - X).max() <= 1e-12 * np.abs(X).max()
        assert np.abs(b_flat.grad[o0:o1].cpu().numpy() - dB).max() <= 1e-12 * np.abs(dB).max()
        got = np.asfortranarray(ga.matrix(i).cpu().numpy()).astype(np.float64)
        assert np.abs(got - dA).max() <= (1e-12 + 2.0 ** -23) * np.abs(dA).max(), n


def test_batched_finite_difference_n64(built):
    """Central difference along an integer direction for a small batch of
    n = 64 matrices whose entries sit on a 2^-12 grid (A +- hE exact)."""
    sizes = np.full(4, 64, np.int32)
    rng = np.random.default_rng(21)
    layout = MatrixBatch(sizes, align=4)
    for i in range(4):
        q = rng.integers(-4 << 12, 4 << 12, size=(64, 64)).astype(np.float64) / 4096
        q[np.diag_indices(64)] += 64
        layout.matrix(i).copy_(torch.from_numpy(q.astype(np.float32)))
    plan = BatchPlan(sizes, outer=rb.FP32)
    rhs = RhsBatch(sizes, 1)
    b = torch.from_numpy(rng.standard_normal(rhs.data.numel())).cuda()
    w = torch.from_numpy(rng.standard_normal(rhs.data.numel())).cuda()
    E = torch.from_numpy(rng.integers(-3, 4, size=layout.data.numel()).astype(np.float32)).cuda()
    h = 2.0 ** -10

    def loss(flat):
        return float((batched_lu_solve(flat, b, layout, plan, refine_iters=3) * w).sum())

    fd = (loss(layout.data + h * E) - loss(layout.data - h * E)) / (2 * h)
    a = layout.data.clone().requires_grad_(True)
    (batched_lu_solve(a, b, layout, plan, refine_iters=3) * w).sum().backward()
    an = float((a.grad.double() * E.double()).sum())
    assert abs(fd - an) <= 1e-5 * max(abs(an), 1e-3), (fd, an)
