/* TEST INFRASTRUCTURE ONLY -- the CPU oracle for the no-pivot LU hot path.
 *
 * This library is a CPU restatement of the reference algorithm (remifa's
 * lu_nopiv_rl / lu_nopiv_inner_rl / lu_nopiv_panel / convert) plus an FP64
 * factorization, the reference's error formulas and the matrix generators.
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
 * load it.  The product library (remifa_b200/liblu_b200.so) never links it.
 *
 * All matrices are column-major; element (i, j) lives at a[i + j*lda].
 *
 * Floating-point order (so results are reproducible bit for bit):
 *   - every "1/d" is an IEEE division, every multiply an IEEE multiply;
 *   - "a -= b*c" inside the panel is the fused fmaf(-b, c, a);
 *   - a GEMM update C -= A*B accumulates acc = fmaf(A[i,t], B[t,j], acc)
 *     for t = 0..K-1 starting from acc = 0, then C = C - acc.
 */
#ifndef LU_B200_ORACLE_H
#define LU_B200_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- generators ------------------------------------------------------ */
/* reference tests/genmat.hxx:69-102 (gen_diagdom): U[-1,1] off-diagonal
 * from std::default_random_engine (default seed), filled row by row, then
 * a_ii = m. */
void orc_gen_diagdom_f32(int64_t m, int64_t n, float* a, int64_t lda);
/* reference tests/common.hxx:298-319 (gen_randmat): U[-1,1], filled column
 * by column, engine seeded with `seed`. */
void orc_gen_randmat_f32(int64_t m, int64_t n, float* a, int64_t lda,
                         uint32_t seed);
/* Counter-based diagonally dominant generator (identical to the library's
 * device generator lu_gen_matrix_c):
 *   kind 0: r_ij = U[-1,1) on a 2^-23 grid;  kind 1: r_ij ~ N(0,1)/sqrt(n)
 *   (Irwin-Hall, 12 terms);  a_ij = r_ij (i != j),
 *   a_ii = alpha * sum_{j != i} |r_ij|;  every entry times 2^kscale;
 *   row i times 2^-round(gamma_bits * i / (n-1)). */
void orc_gen_matrix_f32(int64_t n, float* a, int64_t lda, uint64_t seed,
                        int kind, double alpha, int kscale, double gamma_bits);
/* x ~ U[-1,1) or N(0,1) (kind as above, no 1/sqrt(n)), counter-based. */
void orc_gen_vector_f64(int64_t n, double* x, uint64_t seed, int kind);

/* b = A x with fp32 A and x, accumulated in fp64, rounded once to fp32
 * (reference tests/common.hxx:744-756 calls BLAS sgemv for this). */
void orc_gen_rhs_f32(int64_t m, const float* a, int64_t lda, const float* x,
                     float* b);

/* ---- rounding to the low-precision formats --------------------------- */
/* fmt: 1 = fp16 (RN-even, overflow -> inf), 2 = bf16 (RN-even),
 *      3 = e4m3 (RN-even, saturating to +-448).  Values are returned as the
 *      exactly representable fp32 numbers.  scale_log2 multiplies by
 *      2^scale_log2 before rounding (exact). */
float orc_round_fmt(float x, int fmt, int scale_log2);
void orc_convert(int64_t m, int64_t n, const float* a, int64_t lda, float* out,
                 int64_t ldo, int fmt, int scale_log2);

/* ---- the reference algorithm, restated ------------------------------- */
/* remifa::lu_nopiv_panel<float,8> (src/lu_nopiv.cu:333-400) for an m x n
 * block column (n <= 8) whose diagonal tile copy is d: factors the tile,
 * eliminates the L rows below it and the U columns right of it. */
void orc_panel_f32(int64_t m, int64_t n, const float* d, int64_t ldd, float* l,
                   int64_t ldl, float* u, int64_t ldu);
/* C[m x n] -= A[m x k] * B[k x n] (the reference gemmex with alpha=-1,
 * beta=1), in the accumulation order stated above. */
void orc_gemm_sub_f32(int64_t m, int64_t n, int64_t k, const float* a,
                      int64_t lda, const float* b, int64_t ldb, float* c,
                      int64_t ldc);
/* remifa::lu_nopiv_rl (src/lu_nopiv.hxx:44-208) with ib = 8.
 *   outer_fmt 0: the outer Schur update in fp32 (I = O = FP32);
 *   outer_fmt 1/2/3: the outer update multiplies copies of L21 and U12
 *     rounded to fp16/bf16/e4m3 (TC32 with W = fp32), fp32 accumulation.
 *   outer_fmt 4: split fp16 (new, no reference counterpart): scaled copies
 *     x * 2^s = hi + lo, product hi*hi + hi*lo + lo*hi in fp32.
 *   threads <= 0 uses all OpenMP threads; the result does not depend on the
 *   thread count. */
void orc_lu_rl_f32(int64_t m, int64_t n, int64_t nb, float* a, int64_t lda,
                   int outer_fmt, int threads);
/* Only outer steps [kk0, kk1) of the same factorization (kk1 < 0: to the
 * end); running [0,k) then [k,end) equals one full call. */
void orc_lu_rl_f32_range(int64_t m, int64_t n, int64_t nb, float* a,
                         int64_t lda, int outer_fmt, int threads, int64_t kk0,
                         int64_t kk1);

/* remifa::lu_nopiv_ll (src/lu_nopiv_ll.hxx:41-582) with ib = 8 for W = fp32,
 * I = O = FP32 (the lu_nopiv_ll_f32 wrapper): left-looking outer blocks
 * (one K = ofs update of the block column and block row), left-looking
 * inner tiles (one K = 8t update), then the panel kernel. */
/* lu_nopiv_panel<half,8> with fp16 arithmetic (values held in floats). */
void orc_panel_f16(int64_t m, int64_t n, const float* d, int64_t ldd, float* l,
                   int64_t ldl, float* u, int64_t ldu);
void orc_lu_ll_f32(int64_t m, int64_t n, int64_t nb, float* a, int64_t lda,
                   int threads);
/* Left-looking factorization of an fp16 matrix held in fp32 (fp16-valued
 * entries): fp16 products accumulated in fp32, updated block column / row
 * rounded to fp16, the inner Crout elimination in fp32 rounded to fp16. */
void orc_lu_ll_f16(int64_t m, int64_t n, int64_t nb, float* a, int64_t lda,
                   int threads);
/* Outer blocks wider than `sub` factored as sub-blocks (the product's
 * nesting for nb > 128); panel_fp32: the fp16 variant with OP = OF = fp32. */
void orc_lu_ll_f32_sub(int64_t m, int64_t n, int64_t nb, float* a, int64_t lda,
                       int threads, int64_t sub);
void orc_lu_ll_f16_ex(int64_t m, int64_t n, int64_t nb, float* a, int64_t lda,
                      int threads, int64_t sub, int panel_fp32);

/* ---- FP64 oracle ----------------------------------------------------- */
void orc_lu_f64(int64_t n, double* a, int64_t lda);
/* solve with unit-lower L and upper U stored together (no pivots) */
void orc_lu_solve_f64(int64_t n, const double* lu, int64_t ld, double* b);
void orc_lu_solve_f32(int64_t n, const float* lu, int64_t ld, float* b);
/* solve with fp32 factors in fp64 arithmetic */
void orc_lu_solve_f32f64(int64_t n, const float* lu, int64_t ld, double* b);

/* ---- error metrics --------------------------------------------------- */
/* reference tests/errors.hxx:187-249: ||b-Ax||_inf / (||A||_1 ||x||_inf +
 * ||b||_inf), residual accumulated in fp64 */
double orc_nwerr_f32(int64_t m, const float* a, int64_t lda, const float* b,
                     const float* x);
/* reference tests/errors.hxx:23-182: max_i |b-Ax|_i / (|A||x| + |L||U||x|)_i */
double orc_cwerr_f32(int64_t m, const float* a, int64_t lda, const float* b,
                     const float* x, const float* lu, int64_t ldlu);
/* ||A - L U||_F / ||A||_F for fp32 factors, evaluated in fp64 */
double orc_factor_error_f32(int64_t n, const float* a, int64_t lda,
                            const float* lu, int64_t ldlu);
/* ||b - A x||_inf / (||A||_inf ||x||_inf) with fp32 A and fp64 b, x */
double orc_backward_error_f64(int64_t n, const float* a, int64_t lda,
                              const double* b, const double* x);

int orc_num_threads(void);

#ifdef __cplusplus
}
#endif
#endif
