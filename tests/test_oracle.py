"""CPU tests of the oracle (test infrastructure): rounding against numpy and
torch, generators against the reference's engine semantics, the restated
RL factorization against FP64, the error formulas on known answers, and —
when present — the golden vectors produced by the reference's own code."""
import glob
import os

import numpy as np
import pytest
import torch

import oracle as O

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
U32 = np.finfo(np.float32).eps / 2  # unit roundoff 2^-24


# ---------------------------------------------------------------- rounding

def _edge_values():
    rng = np.random.default_rng(0)
    v = np.concatenate([
        rng.uniform(-2, 2, 4000), rng.uniform(-7e4, 7e4, 1000),
        rng.uniform(-1e-6, 1e-6, 1000), rng.standard_normal(1000) * 1e3,
        np.array([0.0, -0.0, 65504, 65519, 65520, 1e5, 2.0 ** -24, 3 * 2.0 ** -25,
                  1 + 2.0 ** -11, 1 + 3 * 2.0 ** -11, 448, 464, 1e-3, 2.0 ** -9]),
    ]).astype(np.float32)
    return v.reshape(1, -1)


def test_round_fp16_matches_numpy():
    v = _edge_values()
    got = O.round_fmt(v, O.FMT_FP16)
    with np.errstate(over="ignore"):
        want = v.astype(np.float16).astype(np.float32)
    np.testing.assert_array_equal(got, want)


def test_round_bf16_matches_torch():
    v = _edge_values()
    got = O.round_fmt(v, O.FMT_BF16)
    want = torch.from_numpy(v).to(torch.bfloat16).float().numpy()
    np.testing.assert_array_equal(got, want)


def test_round_e4m3_matches_torch_in_range():
    v = _edge_values()
    v = v[np.abs(v) <= 448].reshape(1, -1)
    got = O.round_fmt(v, O.FMT_E4M3)
    want = torch.from_numpy(v).to(torch.float8_e4m3fn).float().numpy()
    np.testing.assert_array_equal(got, want)


def test_round_e4m3_saturates_and_scales():
    v = np.array([[500.0, -1e6, 448.0, 0.1]], np.float32)
    got = O.round_fmt(v, O.FMT_E4M3)
    np.testing.assert_array_equal(got, [[448, -448, 448, 0.1015625]])
    # power-of-two scale is exact: round(x * 2^3)
    got = O.round_fmt(np.array([[0.1]], np.float32), O.FMT_E4M3, 3)
    assert got[0, 0] == np.float32(0.8125)


# ---------------------------------------------------------------- generators

def _minstd_canonical_uniform(seed, count):
    """std::default_random_engine (minstd_rand0) + uniform_real_distribution
    <float>(-1, 1) as libstdc++ defines them (one engine call per draw)."""
    x = seed
    out = []
    r = np.float32(2147483646)  # max - min + 1 of minstd_rand0, as float
    for _ in range(count):
        x = (16807 * x) % 2147483647
        s = np.float32(x - 1) / r
        if s >= np.float32(1):
            s = np.nextafter(np.float32(1), np.float32(0))
        out.append(np.float32(np.float32(2) * s) + np.float32(-1))
    return np.array(out, np.float32)


def test_gen_randmat_matches_engine_restatement():
    a = O.gen_randmat(7, seed=1)
    want = _minstd_canonical_uniform(1, 7 * 7).reshape(7, 7).T  # column order
    np.testing.assert_array_equal(a, want)


def test_gen_diagdom_structure():
    n = 37
    a = O.gen_diagdom(n, lda=40)
    assert O.ld(a) == 40
    np.testing.assert_array_equal(np.diag(a), np.full(n, n, np.float32))
    off = a[~np.eye(n, dtype=bool)]
    assert off.min() >= -1 and off.max() < 1
    # row-by-row filling: row 0 holds the first n draws (diag then overwritten)
    first = _minstd_canonical_uniform(1, n)
    np.testing.assert_array_equal(a[0, 1:], first[1:])
    np.testing.assert_array_equal(a, O.gen_diagdom(n, lda=40))


@pytest.mark.parametrize("kind", [0, 1])
def test_gen_matrix_dominance_exact(kind):
    n = 96
    a = O.gen_matrix(n, seed=3, kind=kind, alpha=1.5)
    a64 = np.array(a, np.float64)
    off = np.abs(a64).sum(axis=1) - np.abs(np.diag(a64))
    ratio = np.abs(np.diag(a64)) / off
    assert np.all(np.abs(ratio - 1.5) < 1e-6)
    np.testing.assert_array_equal(a, O.gen_matrix(n, seed=3, kind=kind, alpha=1.5))
    assert not np.array_equal(a, O.gen_matrix(n, seed=4, kind=kind, alpha=1.5))


def test_gen_matrix_scaling_is_exact_powers_of_two():
    n = 64
    base = O.gen_matrix(n, seed=9, kind=1, alpha=2.0)
    scaled = O.gen_matrix(n, seed=9, kind=1, alpha=2.0, kscale=8, gamma_bits=10.0)
    shifts = np.rint(10.0 * np.arange(n) / (n - 1))
    want = base * (2.0 ** 8) * (2.0 ** -shifts)[:, None]
    np.testing.assert_array_equal(scaled, want.astype(np.float32))


def test_gen_matrix_normal_moments():
    n = 512
    a = O.gen_matrix(n, seed=1, kind=1, alpha=2.0)
    off = a[~np.eye(n, dtype=bool)] * np.sqrt(n)
    assert abs(off.mean()) < 0.01 and abs(off.std() - 1.0) < 0.01


# ---------------------------------------------------------------- algorithm

@pytest.mark.parametrize("n", [1, 7, 8, 9, 63, 64, 65, 200])
@pytest.mark.parametrize("nb", [8, 64, 256])
def test_lu_rl_against_fp64(n, nb):
    # (a 1 x 1 generated matrix has an empty row sum, i.e. a zero pivot)
    a = O.gen_matrix(n, seed=n, kind=0, alpha=2.0) if n > 1 else \
        np.asfortranarray(np.array([[3.0]], np.float32))
    lu = O.lu_rl(a, nb=nb)
    lu64 = O.lu_f64(a)
    err = np.abs(lu - lu64).max() / np.abs(lu64).max()
    assert err <= 4 * n * U32 + 1e-30
    assert O.factor_error(a, lu) <= 10 * n * U32


def test_lu_rl_exact_integer_case():
    # A = L U with small integers: every intermediate is exact in fp32
    L = np.array([[1, 0, 0, 0], [2, 1, 0, 0], [-1, 3, 1, 0], [4, 0, -2, 1]], np.float32)
    U = np.array([[2, 1, -1, 3], [0, 4, 2, 1], [0, 0, 8, -2], [0, 0, 0, 16]], np.float32)
    a = np.asfortranarray(L @ U)
    lu = O.lu_rl(a, nb=8)
    want = np.tril(L, -1) + U
    np.testing.assert_array_equal(lu, want)


def test_lu_rl_thread_count_independent():
    a = O.gen_matrix(300, seed=2, kind=1, alpha=1.2)
    np.testing.assert_array_equal(O.lu_rl(a, nb=64, threads=1),
                                  O.lu_rl(a, nb=64, threads=4))


def test_lu_rl_partial_last_block():
    # n not a multiple of nb or ib exercises the partial tile/outer block
    a = O.gen_matrix(75, seed=5, kind=0, alpha=2.0)
    lu = O.lu_rl(a, nb=32)
    assert O.factor_error(a, lu) <= 10 * 75 * U32


@pytest.mark.parametrize("fmt,tol", [(1, 2e-3), (2, 1e-2), (3, 1e-1)])
def test_lu_rl_lowprec_outer(fmt, tol):
    n = 256
    a = O.gen_matrix(n, seed=11, kind=1, alpha=1.5)
    lu = O.lu_rl(a, nb=64, outer_fmt=fmt)
    fe = O.factor_error(a, lu)
    assert fe < tol * 0.1
    assert O.factor_error(a, O.lu_rl(a, nb=64)) < fe  # rounding costs accuracy


def test_gemm_sub_against_fp64():
    rng = np.random.default_rng(1)
    A = np.asfortranarray(rng.standard_normal((70, 19)).astype(np.float32))
    B = np.asfortranarray(rng.standard_normal((19, 33)).astype(np.float32))
    C = np.asfortranarray(rng.standard_normal((70, 33)).astype(np.float32))
    want = C.astype(np.float64) - A.astype(np.float64) @ B.astype(np.float64)
    got = np.array(C, copy=True, order="F")
    O.gemm_sub(A, B, got)
    assert np.abs(got - want).max() < 19 * 4 * U32 * 8


def test_panel_equals_unblocked_lu_rows():
    # the panel on an m x 8 column + 8 x m row equals the first 8 steps of
    # unblocked LU restricted to those entries
    m = 40
    a = O.gen_matrix(m, seed=7, kind=0, alpha=2.0)
    d = np.asfortranarray(a[:8, :8].copy())
    got = np.array(a, copy=True, order="F")
    O.panel(m, 8, d, got)
    lu64 = O.lu_f64(np.array(a[:, :], np.float64))
    # the L columns 0..7 and U rows 0..7 are final after the panel
    np.testing.assert_allclose(got[:, :8], lu64[:, :8], rtol=0, atol=1e-5)
    np.testing.assert_allclose(got[:8, :], lu64[:8, :], rtol=0, atol=1e-4 * m)


# ---------------------------------------------------------------- errors

def test_error_metrics_known_answers():
    n = 50
    a = O.gen_matrix(n, seed=1, kind=0, alpha=2.0)
    lu = O.lu_rl(a, nb=16)
    x1 = np.ones(n, np.float32)
    b = O.gen_rhs(a, x1)
    x = O.lu_solve_f32(lu, b)
    nw = O.nwerr(a, b, x)
    cw = O.cwerr(a, b, x, lu)
    assert 0 < nw < 10 * U32 * n and 0 < cw < 10 * U32 * n
    # exact solution of an integer system: zero residual
    I = np.asfortranarray(np.eye(4, dtype=np.float32) * 2)
    assert O.nwerr(I, np.full(4, 2, np.float32), np.ones(4, np.float32)) == 0.0
    # fp64 backward error of the fp64 solve is at the fp64 level
    b64 = np.array(a, np.float64) @ np.ones(n)
    x64 = O.lu_solve_f64(O.lu_f64(a), b64)
    assert O.backward_error(a, b64, x64) < 1e-15


# ---------------------------------------------------------------- golden

def _golden(name):
    p = os.path.join(GOLDEN, name)
    if not os.path.exists(p):
        pytest.skip(f"golden fixture {name} not generated yet")
    return np.load(p)


def test_golden_ref_panel_bit_exact():
    g = _golden("ref_panel_48x8.npz")
    a = np.asfortranarray(g["a_in"])
    np.testing.assert_array_equal(a, O.gen_diagdom(48, lda=48))
    d = np.asfortranarray(a[:8, :8].copy())
    got = np.array(a, copy=True, order="F")
    O.panel(48, 8, d, got)
    np.testing.assert_array_equal(got, g["out"])
    assert int(g["stat"][0]) == 8


def test_golden_ref_convert_bit_exact():
    g = _golden("ref_convert_f32_f16.npz")
    np.testing.assert_array_equal(O.round_fmt(g["a_in"], O.FMT_FP16), g["out"])


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "ref_rl_f32_*.npz"))))
def test_golden_ref_rl_f32(path):
    g = np.load(path)
    nn = g["a_in"].shape[0]
    nb = int(path.split("_nb")[1].split(".")[0])
    a = np.asfortranarray(g["a_in"])
    np.testing.assert_array_equal(a, O.gen_diagdom(nn, lda=nn))
    lu = O.lu_rl(a, nb=nb)
    ref = g["lu"]
    # cuBLAS sums the K = 8 / K = nb updates in an unspecified order, so the
    # restatement agrees to a few ulps rather than bit for bit.
    rel = np.abs(lu - ref).max() / np.abs(ref).max()
    assert rel <= 4 * nn * U32
    x1 = np.ones(nn, np.float32)
    b = O.gen_rhs(a, x1)
    e_ref = O.nwerr(a, b, O.lu_solve_f32(np.asfortranarray(ref), b))
    e_orc = O.nwerr(a, b, O.lu_solve_f32(lu, b))
    assert e_orc <= 4 * e_ref + 1e-12 and e_ref <= 4 * e_orc + 1e-12


def test_golden_ref_rl_tc32():
    g = _golden("ref_rl_tc32_n512_nb128.npz")
    a = np.asfortranarray(g["a_in"])
    lu = O.lu_rl(a, nb=128, outer_fmt=O.FMT_FP16)
    ref = g["lu"]
    rel = np.abs(lu - ref).max() / np.abs(ref).max()
    assert rel < 1e-4
    fe_ref, fe_orc = O.factor_error(a, np.asfortranarray(ref)), O.factor_error(a, lu)
    assert fe_orc <= 2 * fe_ref and fe_ref <= 2 * fe_orc


@pytest.mark.parametrize("n,nb", [(7, 8), (64, 16), (200, 64), (257, 128)])
def test_lu_ll_against_fp64(n, nb):
    a = O.gen_matrix(n, seed=n + 1, kind=1, alpha=1.5)
    lu = O.lu_ll(a, nb=nb)
    assert O.factor_error(a, lu) <= 10 * n * U32
    # same factorization as RL up to rounding
    assert np.abs(lu - O.lu_rl(a, nb=nb)).max() <= 8 * n * U32 * np.abs(lu).max()


def test_golden_ref_ll_f32():
    g = _golden("ref_ll_f32_n256_nb64.npz")
    a = np.asfortranarray(g["a_in"])
    np.testing.assert_array_equal(a, O.gen_diagdom(256, lda=256))
    lu = O.lu_ll(a, nb=64)
    ref = g["lu"]
    rel = np.abs(lu - ref).max() / np.abs(ref).max()
    assert rel <= 4 * 256 * U32
    x1 = np.ones(256, np.float32)
    b = O.gen_rhs(a, x1)
    e_ref = O.nwerr(a, b, O.lu_solve_f32(np.asfortranarray(ref), b))
    e_orc = O.nwerr(a, b, O.lu_solve_f32(lu, b))
    assert e_orc <= 4 * e_ref + 1e-12 and e_ref <= 4 * e_orc + 1e-12


@pytest.mark.parametrize("tag,panel_fp32", [("tc32", False), ("tc16", False),
                                            ("tc32_fp32panel", True)])
def test_golden_ref_ll_f16(tag, panel_fp32):
    """Left-looking factorization of an fp16 matrix: the reference's
    lu_nopiv_ll_f16_tc32xtc32 / _tc16xtc16 / _tc32xtc32_fp32xfp32_fp32xfp32
    (src/lu_nopiv_ll.cxx:282, 246, 618) against the oracle's restatement
    with the fp32 elimination this library uses (the reference eliminates in
    fp16 arithmetic for the first two, in fp32 for the third).  Bounds: max
    difference <= 1 u16 of the largest factor entry, backward error and
    ||A - LU|| within 1.5x; with OP = fp32 on both sides at least 95% of the
    factor entries identical."""
    g = _golden(f"ref_ll_f16_{tag}_n256_nb64.npz")
    a = np.asfortranarray(g["a_in"].astype(np.float32))
    np.testing.assert_array_equal(
        a, O.gen_diagdom(256, lda=256).astype(np.float16).astype(np.float32))
    ref = np.asfortranarray(g["lu"].astype(np.float32))
    lu = O.lu_ll(a, nb=64, fp16_storage=True, panel_fp32=panel_fp32)
    assert np.abs(lu - ref).max() <= 2.0 ** -11 * np.abs(ref).max()
    b = O.gen_rhs(a, np.ones(256, np.float32))
    e_r = O.nwerr(a, b, O.lu_solve_f32(ref, b))
    e_o = O.nwerr(a, b, O.lu_solve_f32(lu, b))
    assert e_o <= 1.5 * e_r and e_r <= 1.5 * e_o, (e_o, e_r)
    f_r, f_o = O.factor_error(a, ref), O.factor_error(a, lu)
    assert f_o <= 1.5 * f_r and f_r <= 1.5 * f_o, (f_o, f_r)
    if panel_fp32:
        assert np.mean(lu == ref) >= 0.95


@pytest.mark.parametrize("n,nb", [(300, 256), (520, 192), (257, 512)])
def test_lu_ll_wide_blocks_against_fp64(n, nb):
    """Outer blocks wider than 128 (factored as 128-wide sub-blocks): the
    same factorization as the reference's single Crout loop up to rounding."""
    a = O.gen_matrix(n, seed=n + 2, kind=1, alpha=1.5)
    lu = O.lu_ll(a, nb=nb)
    assert O.factor_error(a, lu) <= 10 * n * U32
    flat = O.lu_ll(a, nb=nb, sub=nb)  # the reference's loop over the whole block
    assert np.abs(lu - flat).max() <= 8 * n * U32 * np.abs(lu).max()
    assert not np.array_equal(lu, flat) or nb <= 128


def test_generator_kind2_condition_family():
    """kind 2 (every off-diagonal entry -|r_ij|, diagonal alpha * row sum):
    an M-matrix whose 2-norm condition is ~1.06 / (alpha - 1) at any n."""
    for n in (256, 512):
        for am1 in (1e-2, 1e-4):
            a = O.gen_matrix(n, seed=7, kind=2, alpha=1.0 + am1)
            A = np.array(a, dtype=np.float64)
            off = A[~np.eye(n, dtype=bool)]
            assert (off <= 0).all()
            k2 = np.linalg.cond(A, 2)
            assert 0.8 / am1 < k2 < 1.3 / am1, (n, am1, k2)


def test_golden_ref_panel_f16_bit_exact():
    """lu_nopiv_panel<half,8> (fp16 arithmetic) restated by the oracle, bit
    for bit against the reference kernel's output."""
    g = _golden("ref_panel_f16_64x8.npz")
    a = np.asfortranarray(g["a_in"].astype(np.float32))
    d = np.asfortranarray(a[:8, :8].copy())
    got = np.array(a, copy=True, order="F")
    O.panel_f16(64, 8, d, got)
    np.testing.assert_array_equal(got, g["out"].astype(np.float32))
