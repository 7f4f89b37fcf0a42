"""Batched persistent LU against the oracle.

Matrix i of a batch is factored exactly as the right-looking algorithm with
outer block NB (its bucket's block width) and inner block 8 factors it: with
FP32 outer updates bit for bit equal to the oracle's restatement
(oracle.lu_rl with that nb), with fp16 tensor-core updates within the
accumulation-order tolerance used for the single-matrix path."""
import numpy as np
import pytest
import torch

import oracle as O
import remifa_b200 as rb
from remifa_b200.batch import BUCKETS, BatchPlan, MatrixBatch, batch_sizes

pytestmark = pytest.mark.gpu
U32 = 2.0 ** -24

EDGE_SIZES = [1, 2, 7, 8, 9, 15, 16, 31, 32, 33, 63, 64, 65, 100, 127, 128, 129,
              200, 255, 256, 257, 300, 383, 448, 511, 512]


def uniform_tuning(nb, outer):
    return {"nb": [nb] * BUCKETS, "outer": [int(outer)] * BUCKETS}


def expected_info(sizes):
    """The generator's 1 x 1 matrix is [0] (an empty off-diagonal row sum):
    a zero pivot in column 1; every other generated matrix is regular."""
    return [1 if int(n) == 1 else 0 for n in sizes]


def host(mats, i):
    return np.asfortranarray(mats.matrix(i).cpu().numpy())


def test_generator_matches_oracle(built):
    sizes = np.array([1, 16, 33, 100, 512], np.int32)
    mats = MatrixBatch(sizes, align=4).generate(seed=5)
    torch.cuda.synchronize()
    for i, n in enumerate(sizes):
        want = O.gen_matrix(int(n), seed=5 + i, kind=0, alpha=1.5)
        assert np.array_equal(host(mats, i), want), n


@pytest.mark.parametrize("nb", [32, 64])
def test_fp32_bit_exact_vs_oracle(built, nb):
    sizes = np.array(EDGE_SIZES, np.int32)
    mats = MatrixBatch(sizes).generate(seed=100)
    plan = BatchPlan(sizes, outer=rb.FP32, tuning=uniform_tuning(nb, rb.FP32))
    info = plan(mats)
    torch.cuda.synchronize()
    assert info.tolist() == expected_info(sizes)
    for i, n in enumerate(sizes):
        a = O.gen_matrix(int(n), seed=100 + i, kind=0, alpha=1.5)
        want = O.lu_rl(a, nb=nb, outer_fmt=0)
        got = host(mats, i)
        assert np.array_equal(got, want), (n, np.abs(got - want).max())


@pytest.mark.parametrize("nb", [32, 64])
def test_tc_vs_oracle(built, nb):
    sizes = np.array(EDGE_SIZES, np.int32)
    mats = MatrixBatch(sizes, align=4).generate(seed=200)
    plan = BatchPlan(sizes, outer=rb.TC32, tuning=uniform_tuning(nb, rb.TC32))
    info = plan(mats)
    torch.cuda.synchronize()
    assert info.tolist() == expected_info(sizes)
    for i, n in enumerate(sizes):
        a = O.gen_matrix(int(n), seed=200 + i, kind=0, alpha=1.5)
        want = O.lu_rl(a, nb=nb, outer_fmt=O.FMT_FP16)
        got = host(mats, i)
        if n <= nb:  # one block column: no outer update, pure FP32 elimination
            assert np.array_equal(got, want), n
            continue
        rel = np.abs(got - want).max() / np.abs(want).max()
        assert rel < 64 * n * U32, (n, rel)
        fe_g, fe_o = O.factor_error(a, got), O.factor_error(a, want)
        assert fe_g <= 2 * fe_o + 1e-7 and fe_o <= 2 * fe_g + 1e-7, (n, fe_g, fe_o)


def test_mixed_buckets_and_padding(built):
    """Per-bucket block widths and precisions in one launch, padded lda."""
    sizes = np.array([20, 40, 80, 160, 320, 512, 24, 48, 96, 192, 384], np.int32)
    tuning = {"nb": [32, 64, 32, 64, 32, 64],
              "outer": [int(rb.FP32), int(rb.TC32), int(rb.FP32), int(rb.TC32),
                        int(rb.TC32), int(rb.FP32)]}
    mats = MatrixBatch(sizes, align=8).generate(seed=300)
    plan = BatchPlan(sizes, outer=rb.TC32, tuning=tuning)
    assert plan.tuning() == tuning
    plan(mats)
    torch.cuda.synchronize()
    for i, n in enumerate(sizes):
        b = rb.batch.bucket_of(int(n))
        nb, outer = tuning["nb"][b], tuning["outer"][b]
        a = O.gen_matrix(int(n), seed=300 + i, kind=0, alpha=1.5)
        got = host(mats, i)
        if outer == int(rb.FP32):
            assert np.array_equal(got, O.lu_rl(a, nb=nb, outer_fmt=0)), n
        else:
            want = O.lu_rl(a, nb=nb, outer_fmt=O.FMT_FP16)
            assert np.abs(got - want).max() / np.abs(want).max() < 64 * n * U32, n


def test_graph_replay_matches_direct_call(built):
    sizes = batch_sizes(600, seed=3)
    ref = MatrixBatch(sizes).generate(seed=9)
    plan = BatchPlan(sizes, outer=rb.TC32)
    plan(ref)
    mats = MatrixBatch(sizes).generate(seed=9)
    info = torch.zeros(len(sizes), dtype=torch.int32, device="cuda")
    g = plan.graph(mats, info)
    torch.cuda.synchronize()
    for _ in range(2):
        mats.generate(seed=9)
        g.launch()
        torch.cuda.synchronize()
        assert torch.equal(mats.data, ref.data)
        assert int(info.abs().sum()) == 0
    g.close()


def test_zero_pivot_reports_column(built):
    sizes = np.array([40, 100, 300], np.int32)
    mats = MatrixBatch(sizes).generate(seed=4)
    m = mats.matrix(1)
    m[:, :] = torch.eye(100, device="cuda")
    m[57, 57] = 0.0
    plan = BatchPlan(sizes, outer=rb.TC32)
    info = plan(mats)
    torch.cuda.synchronize()
    assert info.tolist() == [0, 58, 0]


def test_autotune_returns_valid_table_and_keeps_parity(built):
    sizes = batch_sizes(2000, seed=11)
    plan = BatchPlan(sizes, outer=rb.TC32)
    t = plan.autotune(reps=2)
    assert all(nb in (32, 64) for nb in t["nb"])
    assert all(o == int(rb.TC32) for o in t["outer"])
    assert plan.tuning() == t
    mats = MatrixBatch(sizes).generate(seed=11)
    info = plan(mats)
    torch.cuda.synchronize()
    assert int(info.abs().sum()) == 0
    for i in range(0, len(sizes), 97):
        n = int(sizes[i])
        nb = t["nb"][rb.batch.bucket_of(n)]
        a = O.gen_matrix(n, seed=11 + i, kind=0, alpha=1.5)
        want = O.lu_rl(a, nb=nb, outer_fmt=O.FMT_FP16)
        got = host(mats, i)
        assert np.abs(got - want).max() / np.abs(want).max() < 64 * n * U32, n


def test_full_batch_10000_backward_error(built):
    """The C4 workload: 10,000 log-uniform sizes in [16, 512); every info 0
    and ||A - LU|| / ||A|| at the fp16-update level on a sample."""
    sizes = batch_sizes(10_000, seed=11)
    mats = MatrixBatch(sizes).generate(seed=11)
    plan = BatchPlan(sizes, outer=rb.TC32)
    info = plan(mats)
    torch.cuda.synchronize()
    assert int(info.abs().sum()) == 0
    nb = plan.tuning()["nb"]
    for i in range(0, 10_000, 499):
        n = int(sizes[i])
        a = O.gen_matrix(n, seed=11 + i, kind=0, alpha=1.5)
        fe = O.factor_error(a, host(mats, i))
        fe_o = O.factor_error(a, O.lu_rl(a, nb=nb[rb.batch.bucket_of(n)],
                                         outer_fmt=O.FMT_FP16))
        assert fe <= 2 * fe_o + 1e-7, (n, fe, fe_o)
