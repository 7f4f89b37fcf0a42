/*
 * lu_b200.h -- C ABI of the B200-native no-pivot LU library (liblu_b200.so).
 *
 * Drop-in boundary for the lu_nopiv entry points of flipflapflop/remifa.
 * Every function is plain C: device pointers are void*, sizes are int64_t,
 * streams are CUDA streams, nothing throws.  All matrices are column-major
 * (element (i, j) at a[i + j*lda]).  Factorizations are in place: the strict
 * lower triangle holds the unit-lower L, the upper triangle holds U, and no
 * pivoting is performed.
 *
 * Each entry point names the reference interface (file:line, paths inside
 * the reference project) that it replaces.  include/remifa_shim.hxx (and the
 * headers with the reference's file names in include/remifa/) maps the
 * reference's C++ templates and wrappers onto these.
 */
#ifndef LU_B200_H
#define LU_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LU_B200_ABI_VERSION 1

#if defined(__GNUC__)
#define LU_API __attribute__((visibility("default")))
#else
#define LU_API
#endif

/* Same type as cudaStream_t / CUstream (an opaque driver handle). */
typedef struct CUstream_st* lu_stream_t;

typedef enum lu_status {
  LU_SUCCESS = 0,
  LU_ERR_INVALID_ARG = 1,   /* bad size, leading dimension, pointer or option */
  LU_ERR_CUDA = 2,          /* a CUDA runtime/driver call failed */
  LU_ERR_ALLOC = 3,         /* device allocation failed */
  LU_ERR_UNSUPPORTED = 4,   /* valid but unimplemented combination */
  LU_ERR_WORKSPACE = 5,     /* caller workspace too small */
  LU_ERR_NOT_CONVERGED = 6, /* iterative refinement did not reach its target */
  LU_ERR_TIMEOUT = 7,       /* a bounded device-side wait gave up */
  LU_ERR_NO_DEVICE = 8      /* no usable sm_100 device */
} lu_status;

/* Storage types. */
typedef enum lu_dtype {
  LU_F32 = 0,
  LU_F16 = 1,
  LU_BF16 = 2,
  LU_E4M3 = 3,
  LU_F64 = 4
} lu_dtype;

/* Update compute types.  0..3 keep the reference's enum values
 * (remifa::compute_type, src/utils.hxx:18-24); 4..6 are new tensor-core
 * update kinds (operands rounded as named, fp32 accumulation). */
typedef enum lu_compute {
  LU_COMPUTE_FP32 = 0,       /* SIMT fp32, fp32 accumulation */
  LU_COMPUTE_FP16 = 1,       /* fp16 in, fp16 out (W = fp16 only) */
  LU_COMPUTE_TC32 = 2,       /* tensor cores: fp16 operands, fp32 accumulate */
  LU_COMPUTE_TC16 = 3,       /* tensor cores: fp16 operands, fp16 result */
  LU_COMPUTE_TC32_BF16 = 4,  /* tensor cores: bf16 operands, fp32 accumulate */
  LU_COMPUTE_TC32_E4M3 = 5,  /* tensor cores: e4m3 operands with a power-of-two
                                scale per 128-row / 128-column tile */
  LU_COMPUTE_TC32_SPLIT = 6  /* compensated split fp16: hi*hi + hi*lo + lo*hi */
} lu_compute;

typedef enum lu_variant {
  LU_RIGHT_LOOKING = 0, /* remifa::lu_nopiv_rl (src/lu_nopiv.hxx:44-208) */
  LU_LEFT_LOOKING = 1   /* remifa::lu_nopiv_ll (src/lu_nopiv_ll.hxx:41-582) */
} lu_variant;

typedef struct lu_opts {
  int64_t nb;           /* outer block size (reference runtime nb, default 256) */
  int32_t ib;           /* inner block size: 8 (the reference's compile-time ib) */
  int32_t inner_update; /* lu_compute for updates inside the outer block */
  int32_t outer_update; /* lu_compute for the trailing (Schur) update */
  int32_t variant;      /* lu_variant */
  int32_t lookahead;    /* 1: factor panel k+1 while update k runs */
  int32_t diag_width;   /* width of the one-CTA diagonal factorization
                           (multiple of 8, <= 128; 0 = default 128) */
  int32_t panel_fp32;   /* fp16 storage, left-looking: 1 keeps each block
                           column / row update in fp32 until its panel is
                           factored (the reference's OP = OF = fp32 wrappers,
                           src/lu_nopiv_ll.hxx:172-201); 0 rounds the update
                           to fp16 first (OP = fp16).  Ignored for fp32 storage. */
  int32_t bulk_steps;   /* right-looking with look-ahead and fp16 / bf16 trailing
                           updates: q = 2 .. 8 consecutive outer steps'
                           updates of the bulk of the trailing matrix in one
                           pass (C - (L_k U_k + ... + L_k+q-1 U_k+q-1), one
                           fp32 accumulator, C read and written once per q
                           steps); 0 = the default, 4; 1 applies every step
                           separately, the reference's rounding order.
                           Ignored elsewhere. */
  int32_t reserved[6];
} lu_opts;

/* Defaults: nb = 256, ib = 8, FP32/FP32, right-looking, look-ahead on. */
LU_API void lu_opts_default(lu_opts* opts);

LU_API const char* lu_status_string(lu_status s);
LU_API int lu_abi_version(void);
/* Message of the last CUDA failure seen by this thread (empty if none). */
LU_API const char* lu_last_error(void);

/* Bytes of device workspace lu_nopiv_rl_c / lu_nopiv_ll_c need for these
 * arguments (replaces the reference's internal cudaMalloc,
 * src/lu_nopiv.hxx:111 and src/lu_nopiv_ll.hxx:162-190). */
LU_API lu_status lu_workspace_size(const lu_opts* opts, int64_t m, int64_t n,
                            lu_dtype dtype_a, size_t* bytes);

/* In-place no-pivot LU, right-looking.
 * Replaces remifa::lu_nopiv_rl<T,I,O,ib,use_cutlass,CpyType>
 * (src/lu_nopiv.hxx:44-63).
 *   m, n      : matrix size (square: m == n, as the reference's inner loop
 *               assumes, src/lu_nopiv_inner_rl.hxx:124-129)
 *   d_a, lda  : device matrix of type dtype_a (LU_F32 or LU_F16)
 *   d_info    : device int; 0 on success, k > 0 if the k-th pivot (1-based)
 *               was zero or not finite (the factorization still completes)
 *   d_a_lowp  : optional fp16 m x n buffer (ld_lowp); when given it receives
 *               the fp16 copy of the factors the reference leaves in its
 *               d_a_cpy argument.  Unlike the reference it is never required.
 *   workspace : device memory of lu_workspace_size bytes, or NULL to let the
 *               library allocate stream-ordered memory (cudaMallocAsync).
 * Asynchronous with respect to the host: work is queued on `stream`; call
 * cudaStreamSynchronize before reading d_a. */
LU_API lu_status lu_nopiv_rl_c(const lu_opts* opts, lu_stream_t stream, int64_t m,
                        int64_t n, void* d_a, lu_dtype dtype_a, int64_t lda,
                        int* d_info, void* d_a_lowp, int64_t ld_lowp,
                        void* workspace, size_t ws_bytes);

/* The right-looking factorization of an fp32 matrix in host memory (new; the
 * reference takes device pointers only).  h_a (n x n, lda) is copied into
 * the device buffer d_a (ldda) by column chunks of whole outer blocks on an
 * internal copy stream; each chunk, once in, receives the outer steps of the
 * earlier chunks (beside the factorization of the previous chunk), sends
 * its rows above the chunk (final by then) back into h_a on a second
 * internal copy stream, then runs its own steps, each of which sends the
 * rest of its finished block column back the same way -- so both transfers
 * overlap the factorization.  The factors are bit-identical to
 * lu_nopiv_rl_c's.  With look-ahead and tensor-core updates two extra
 * operand buffers (each the size of one packed L21 / U12 pair) are taken
 * from cudaMallocAsync on `stream` besides the workspace.  h_a should be pinned host memory (cudaHostAlloc /
 * cudaHostRegister) for the copies to run asynchronously.  d_info as for
 * lu_nopiv_rl_c.  Asynchronous: synchronise `stream` before reading h_a. */
LU_API lu_status lu_nopiv_rl_host_c(const lu_opts* opts, lu_stream_t stream, int64_t n,
                                    float* h_a, int64_t lda, float* d_a, int64_t ldda,
                                    int* d_info, void* workspace, size_t ws_bytes);

/* In-place no-pivot LU, left-looking (Crout).
 * Replaces remifa::lu_nopiv_ll<...> (src/lu_nopiv_ll.hxx:41-66) and its 30
 * wrappers lu_nopiv_ll_* (src/lu_nopiv_ll.hxx:586-793). Arguments as
 * lu_nopiv_rl_c. */
LU_API lu_status lu_nopiv_ll_c(const lu_opts* opts, lu_stream_t stream, int64_t m,
                        int64_t n, void* d_a, lu_dtype dtype_a, int64_t lda,
                        int* d_info, void* d_a_lowp, int64_t ld_lowp,
                        void* workspace, size_t ws_bytes);

/* Panel kernel: factors the n x n (n <= 8) diagonal tile whose copy is d,
 * applies it to the m - n rows below (L, in l) and the m - n columns to its
 * right (U, in u).  stat receives n.
 * Replaces remifa::lu_nopiv_panel<T,8> (src/lu_nopiv.cuh:12-19,
 * src/lu_nopiv.cu:364-400).  dtype: LU_F32 or LU_F16. */
LU_API lu_status lu_panel_c(lu_stream_t stream, lu_dtype dtype, int64_t m, int64_t n,
                     const void* d, int64_t ldd, void* l, int64_t ldl, void* u,
                     int64_t ldu, int* stat);

/* Cast copy out = round(a * 2^scale_log2), m x n column-major.
 * Replaces remifa::convert<TA,TAO> (src/convert.cuh:17-18,
 * src/convert.cu:324-387).  Supported (in -> out): f32 -> f16/bf16/e4m3/f32,
 * f16 -> f32, f64 -> f16, f16 -> f64, f32 -> f64, f64 -> f32.  Rounding is
 * to nearest even; e4m3 saturates to +-448. */
LU_API lu_status lu_convert_c(lu_stream_t stream, int64_t m, int64_t n, const void* a,
                       lu_dtype type_a, int64_t lda, void* out,
                       lu_dtype type_out, int64_t ldout, int scale_log2);

/* C = alpha * A * B + beta * C (no transposes), A m x k, B k x n.
 * Replaces remifa::gemmex<Impl,Op,Acc,In,Out> (src/gemm.cuh:24-40,
 * src/gemm.cu:17-316) without cuBLAS:
 *   LU_COMPUTE_FP32 : A, B, C fp32; SIMT fp32.  With alpha = -1, beta = 1
 *                     the result is C - sum_t fma-chain(A[i,t] B[t,j]).
 *   LU_COMPUTE_TC32 / _BF16 / _E4M3 / _SPLIT : A, B fp32 (rounded on the
 *                     fly to the operand type by the library), C fp32,
 *                     tcgen05 tensor cores, fp32 accumulation.
 * workspace/ws_bytes: scratch for the rounded operand copies (NULL: the
 * library allocates stream-ordered memory). */
LU_API lu_status lu_gemm_update_c(lu_stream_t stream, lu_compute compute, int64_t m,
                           int64_t n, int64_t k, double alpha, const void* a,
                           int64_t lda, const void* b, int64_t ldb,
                           double beta, void* c, int64_t ldc, void* workspace,
                           size_t ws_bytes);

/* lu_gemm_update_c with the storage types of A, B (both LU_F32 or both
 * LU_F16) and C (LU_F32 or LU_F16): the reference's gemmex instantiations
 * with fp16 operands (src/gemm.cu:17-316).
 *   LU_COMPUTE_FP32 : fp32 A, B, C only (SIMT).
 *   LU_COMPUTE_TC32 : fp16 (or fp32, rounded to fp16) A, B; C fp32 or fp16
 *                     (C = rn16(C + alpha * acc) with acc and the sum in fp32).
 *   LU_COMPUTE_TC16, LU_COMPUTE_FP16 : as TC32 (the reference accumulates in
 *                     fp16; the tensor cores here accumulate in fp32 and round
 *                     the result once).
 *   the other tensor-core kinds: fp32 A, B, C as lu_gemm_update_c.
 * Tensor-core kinds need beta = 1. */
LU_API lu_status lu_gemm_update_ex_c(lu_stream_t stream, lu_compute compute, int64_t m,
                                     int64_t n, int64_t k, double alpha, const void* a,
                                     lu_dtype type_a, int64_t lda, const void* b,
                                     lu_dtype type_b, int64_t ldb, double beta, void* c,
                                     lu_dtype type_c, int64_t ldc, void* workspace,
                                     size_t ws_bytes);

/* Seeded, counter-based test-matrix generator (bit-identical to the CPU
 * oracle): kind 0: r_ij = U[-1,1); kind 1: r_ij ~ N(0,1)/sqrt(n);
 * a_ii = alpha * sum_{j!=i} |r_ij|; all entries * 2^kscale; row i scaled by
 * 2^-round(gamma_bits * i / (n-1)).  New: the reference generates on the host
 * (tests/genmat.hxx:69-102). */
LU_API lu_status lu_gen_matrix_c(lu_stream_t stream, int64_t n, float* d_a,
                          int64_t lda, uint64_t seed, int kind, double alpha,
                          int kscale, double gamma_bits);

/* Equilibration in place by powers of two: LAPACK geequb's row / column
 * scales and laqge's decision (rows when rowcnd < 0.1 or amax is outside
 * the safe range, columns when colcnd < 0.1), as the reference applies them
 * on the host before factoring (tests/testing_lu_gpu.hxx:288-311); force =
 * 1 applies both scalings whatever laqge decides (a matrix scaled as a whole
 * by a large power of two keeps rowcnd = colcnd = 1, yet its entries may lie
 * outside the fp16 range of the tensor-core operands).  d_a
 * (fp32, n x n) becomes R A C; d_r / d_c (device, n floats) receive the
 * diagonals of R and C (ones where not applied); *equed (host) 'N', 'R',
 * 'C' or 'B'; *rowcnd / *colcnd / *amax (host, may be NULL) geequb's ratios
 * and max |a_ij|.  Every scale is a power of two, so R A C is exact and
 * A x = b becomes (R A C) y = R b with x = C y.  Synchronises the stream
 * (the decision is taken on the host). */
LU_API lu_status lu_equilibrate_c(lu_stream_t stream, int64_t n, float* d_a, int64_t lda,
                                  float* d_r, float* d_c, int force, char* equed,
                                  double* rowcnd, double* colcnd, double* amax);

/* ---- solve and iterative refinement (new: the reference solves on the
 * host with LAPACK getrs, tests/testing_lu_gpu.hxx:1309-1313) ------------ */

/* op(A) X = B with the in-place factors of A (fp32, ldlu): trans = 0 solves
 * L U X = B, trans = 1 solves (L U)^T X = B.  d_x (fp64, n x nrhs, ldx)
 * holds B on entry and X on exit.  fp64 arithmetic throughout.  One launch
 * per triangle; a few counter words come from cudaMallocAsync on the
 * stream (lu_refine_c and lu_refine_static_c take them from their own
 * scratch instead). */
LU_API lu_status lu_solve_c(lu_stream_t stream, int64_t n, const float* d_lu,
                            int64_t ldlu, double* d_x, int64_t ldx,
                            int64_t nrhs, int trans);

/* Bytes of device workspace lu_refine_c needs for size n. */
LU_API lu_status lu_refine_workspace_size(int64_t n, size_t* bytes);

/* FP64 iterative refinement of A x = b (A fp32, the original matrix; d_lu
 * its factors, mixed precision allowed).  x0 = (LU)^-1 b; then repeatedly
 * r = b - A x in fp64, berr = ||r||inf / (||A||inf ||x||inf + ||b||inf),
 * stop when berr <= tol, else x += (LU)^-1 r, at most max_iter updates.
 * Synchronises the stream once per iteration to read berr.  *iters and
 * *berr (host pointers, may be NULL) receive the iteration count and the
 * final backward error; returns LU_ERR_NOT_CONVERGED if tol was not met. */
LU_API lu_status lu_refine_c(lu_stream_t stream, int64_t n, const float* d_a,
                             int64_t lda, const float* d_lu, int64_t ldlu,
                             const double* d_b, double* d_x, double tol,
                             int max_iter, int* iters, double* berr,
                             void* workspace, size_t ws_bytes);

/* lu_refine_c without any allocation (no counterpart in the reference): the
 * scratch is one array compiled into the library (LU_REFINE_STATIC_SCRATCH_BYTES
 * of device memory per device), so n <= LU_REFINE_STATIC_MAX_N, else
 * LU_ERR_INVALID_ARG with nothing enqueued.  For callers that cannot hand
 * over or allocate device memory.  Arguments are checked as lu_refine_c
 * checks them, before any device call.  The first call on a device (and the
 * first after cudaDeviceReset) looks the array up (cudaGetSymbolAddress).
 * Like lu_refine_c it synchronises the stream once per iteration, so it must
 * not be called while the stream is being captured.  Calls overlapping in
 * time on one device share the array and race. */
#define LU_REFINE_STATIC_MAX_N 4096
#define LU_REFINE_STATIC_SCRATCH_BYTES 614400
LU_API lu_status lu_refine_static_c(lu_stream_t stream, int64_t n, const float* d_a,
                                    int64_t lda, const float* d_lu, int64_t ldlu,
                                    const double* d_b, double* d_x, double tol,
                                    int max_iter, int* iters, double* berr);

/* GMRES-based FP64 refinement (GMRES-IR; new): each correction A d = r is
 * solved by restarted GMRES on (LU)^-1 A d = (LU)^-1 r in fp64 (classical
 * Gram-Schmidt applied twice; at most `restart` Arnoldi steps per outer
 * iteration, fewer once the GMRES residual estimate falls below inner_tol
 * times its start), which converges where classic refinement stalls
 * (kappa(A) times the factors' relative error >= 1: fp16 / bf16 / e4m3
 * factors of ill-conditioned matrices).  Stops when the backward error
 * ||r||inf / (||A||inf ||x||inf + ||b||inf) <= tol or after max_outer
 * outer iterations (LU_ERR_NOT_CONVERGED then).  *outer_iters / *inner_iters
 * / *berr (host, may be NULL): outer iterations, Arnoldi steps in total,
 * the final backward error.  Synchronises the stream once per Arnoldi step.
 * Workspace: lu_gmres_ir_workspace_size (or NULL: stream-ordered). */
#define LU_GMRES_MAX_RESTART 60
LU_API lu_status lu_gmres_ir_workspace_size(int64_t n, int restart, size_t* bytes);
LU_API lu_status lu_gmres_ir_c(lu_stream_t stream, int64_t n, const float* d_a, int64_t lda,
                               const float* d_lu, int64_t ldlu, const double* d_b,
                               double* d_x, double tol, int max_outer, int restart,
                               double inner_tol, int* outer_iters, int* inner_iters,
                               double* berr, void* workspace, size_t ws_bytes);

/* Several right-hand sides (B, X fp64, n x nrhs) and the transposed system
 * (trans = 1: A^T X = B, backward error with ||A||_1).  All columns are
 * refined together (one multi-column solve per iteration) until the largest
 * backward error over the columns is <= tol; *iters / *berr receive the
 * iteration count and that largest backward error.  Workspace:
 * lu_refine_ex_workspace_size (or NULL for stream-ordered allocation). */
LU_API lu_status lu_refine_ex_workspace_size(int64_t n, int64_t nrhs, size_t* bytes);
LU_API lu_status lu_refine_ex_c(lu_stream_t stream, int64_t n, int64_t nrhs,
                                const float* d_a, int64_t lda, const float* d_lu,
                                int64_t ldlu, const double* d_b, int64_t ldb,
                                double* d_x, int64_t ldx, int trans, double tol,
                                int max_iter, int* iters, double* berr,
                                void* workspace, size_t ws_bytes);

/* ---- adjoint of the solve (new) ---------------------------------------- */

/* Backward pass of X = A^-1 B for a loss with gradient G = dL/dX, reusing
 * the forward factors d_lu of A: on exit d_g holds dL/dB = A^-T G and, when
 * d_da is not NULL, d_da = dL/dA = -(A^-T G) X^T (fp64 outer product stored
 * fp32); d_x is the forward solution X (fp64, n x nrhs).
 * d_a == NULL: A^-T G by two transposed triangular solves (U^T, then L^T).
 * d_a != NULL (the fp32 matrix A): FP64 refinement of A^T dB = G to tol as in
 * lu_refine_ex_c (trans = 1); LU_ERR_NOT_CONVERGED is returned after dA is
 * still written.  Workspace: lu_adjoint_workspace_size, or NULL for
 * stream-ordered allocation; unused without refinement. */
LU_API lu_status lu_adjoint_workspace_size(int64_t n, int64_t nrhs, size_t* bytes);
LU_API lu_status lu_adjoint_c(lu_stream_t stream, int64_t n, int64_t nrhs,
                              const float* d_a, int64_t lda, const float* d_lu,
                              int64_t ldlu, const double* d_x, int64_t ldx,
                              double* d_g, int64_t ldg, float* d_da, int64_t ldda,
                              double tol, int max_iter, int* iters, double* berr,
                              void* workspace, size_t ws_bytes);

/* ---- batched factorization of many uneven matrices (new) -------------- */

/* Many independent no-pivot LUs (fp32, column-major, in place, sizes 1 ..
 * LU_BATCH_MAX_N) in one persistent launch.  A plan fixes the sizes and the
 * per-size-bucket choice of block width (32 or 64) and outer-update
 * precision (LU_COMPUTE_FP32 or LU_COMPUTE_TC32); executing it allocates
 * nothing, so the launch can be captured in a CUDA graph (lu_batch_graph_*).
 * Matrix i is factored exactly as lu_nopiv_rl_c with nb = its bucket's block
 * width and inner updates FP32 would factor it.  Buckets: n < 32, [32, 64),
 * [64, 128), [128, 256), [256, 512), 512. */
#define LU_BATCH_MAX_N 512
#define LU_BATCH_BUCKETS 6
typedef struct lu_batch_tuning {
  int32_t nb[LU_BATCH_BUCKETS];     /* 32 or 64 */
  int32_t outer[LU_BATCH_BUCKETS];  /* LU_COMPUTE_FP32 or LU_COMPUTE_TC32 */
} lu_batch_tuning;
typedef struct lu_batch_plan_t* lu_batch_plan;
typedef struct lu_batch_graph_t* lu_batch_graph;

/* opts: inner_update FP32; outer_update FP32 or TC32 (every bucket's
 * default); nb 0 (= 64), 32 or 64.  tuning (optional) overrides per bucket.
 * h_n: host array of the batch sizes.  Allocates the plan's device arrays
 * on the current device. */
LU_API lu_status lu_batch_plan_create(const lu_opts* opts, int64_t batch,
                                      const int32_t* h_n, const lu_batch_tuning* tuning,
                                      lu_batch_plan* plan);
LU_API void lu_batch_plan_destroy(lu_batch_plan plan);
LU_API lu_status lu_batch_plan_tuning(lu_batch_plan plan, lu_batch_tuning* out);
LU_API lu_status lu_batch_plan_set_tuning(lu_batch_plan plan, const lu_batch_tuning* t);

/* Factor matrix i at d_ptrs[i] (device array of device pointers) with
 * leading dimension d_lda[i] (device array; NULL: lda = n_i) in place;
 * d_info[i] = 0, the 1-based column of the first zero / non-finite pivot,
 * or -1 if a bounded device wait gave up.  Asynchronous on `stream`. */
LU_API lu_status lu_batch_c(lu_batch_plan plan, lu_stream_t stream, float* const* d_ptrs,
                            const int32_t* d_lda, int32_t* d_info);

/* Project autotuner: for every size bucket present in the plan, times each
 * block width (32, 64) at the plan's outer precision on up to 4 x SMs
 * seeded matrices with that bucket's sizes (median of `reps` runs after a
 * warm-up), keeps the fastest in the plan and returns the table in *out
 * (may be NULL).  Allocates and synchronises: a setup-time call. */
LU_API lu_status lu_batch_autotune(lu_batch_plan plan, lu_stream_t stream, int reps,
                                   lu_batch_tuning* out);

/* The same call captured once into a CUDA graph and replayed. */
LU_API lu_status lu_batch_graph_create(lu_batch_plan plan, lu_stream_t stream,
                                       float* const* d_ptrs, const int32_t* d_lda,
                                       int32_t* d_info, lu_batch_graph* graph);
LU_API lu_status lu_batch_graph_launch(lu_batch_graph graph, lu_stream_t stream);
LU_API void lu_batch_graph_destroy(lu_batch_graph graph);

/* Solve with the factors of every matrix of the plan: d_x[i] (device, fp64,
 * n_i x nrhs, ld n_i) holds B_i on entry and X_i = op(A_i)^-1 B_i on exit
 * (trans = 1: A_i^T).  fp32 factors d_lu[i] (ld d_ldlu[i], NULL: n_i), fp64
 * arithmetic; with the original matrices d_a (ld d_lda, NULL: n_i) each
 * column then gets refine_iters rounds of FP64 refinement.  One warp per
 * (matrix, column), no allocation, asynchronous. */
LU_API lu_status lu_batch_solve_c(lu_batch_plan plan, lu_stream_t stream,
                                  const float* const* d_lu, const int32_t* d_ldlu,
                                  const float* const* d_a, const int32_t* d_lda,
                                  double* const* d_x, int32_t nrhs, int trans,
                                  int refine_iters);

/* Backward pass of X_i = A_i^-1 B_i for the whole batch: d_g[i] (dL/dX_i,
 * fp64 n_i x nrhs) is overwritten with dL/dB_i = A_i^-T G_i (refined as in
 * lu_batch_solve_c), and d_da[i] (fp32, ld d_ldda[i] or n_i; may be NULL)
 * receives dL/dA_i = -(A_i^-T G_i) X_i^T.  d_x: the forward solutions. */
LU_API lu_status lu_batch_adjoint_c(lu_batch_plan plan, lu_stream_t stream,
                                    const float* const* d_lu, const int32_t* d_ldlu,
                                    const float* const* d_a, const int32_t* d_lda,
                                    double* const* d_x, double* const* d_g,
                                    float* const* d_da, const int32_t* d_ldda,
                                    int32_t nrhs, int refine_iters);

/* Seeded generator for a batch: matrix i is lu_gen_matrix_c(n_i, seed + i,
 * kind, alpha) (no scaling).  d_n, d_lda (NULL: lda = n): device arrays. */
LU_API lu_status lu_gen_batch_c(lu_stream_t stream, int64_t batch, float* const* d_ptrs,
                                const int32_t* d_n, const int32_t* d_lda, uint64_t seed,
                                int kind, double alpha);

/* Self-check (no reference counterpart): counts, over all 2^32 float bit
 * patterns, the inputs where the library's correctly rounded reciprocal
 * (used for the 1/d of every pivot) differs from CUDA's __frcp_rn; writes
 * the count to *d_bad (device).  Expected 0. */
LU_API lu_status lu_selfcheck_rcp_c(lu_stream_t stream, unsigned long long* d_bad);

/* ---- self-tests of the bounded device waits (new) ----------------------
 * Every cross-role or cross-CTA wait in the library's kernels is bounded;
 * these entry points make such waits run out on purpose, by construction,
 * so the give-up path can be tested without a fault or a hang. */
#define LU_SELFTEST_SCRATCH_BYTES (2 << 20)

/* The tensor-core update (fp16 operands, 512 x 512 x 64) with its TMA
 * producer withheld: no loads are issued, so every consumer wait runs out
 * after wait_cycles clock cycles.  streaming = 1 selects the epilogue that
 * streams C in by TMA (its C loads are then in flight when the waits give
 * up and must be drained), 0 the reduce-add epilogue.  d_scratch: device,
 * 1024-byte aligned, LU_SELFTEST_SCRATCH_BYTES.  On completion d_out[0]
 * (device int) holds the kernel's error code (non-zero: a wait gave up) and
 * d_out[1] the info a factorization reports for it (-1). */
LU_API lu_status lu_selftest_wait_update_c(lu_stream_t stream, long long wait_cycles,
                                           int streaming, void* d_scratch, size_t bytes,
                                           int* d_out);

/* The forward solve L x = b (unit lower factor d_lu, n >= 128; x fp64 holds b
 * on entry) with the row block solved first withholding its solution, each
 * wait bounded by wait_ns nanoseconds: the waits for it run out, x ends with
 * NaN, *d_expired (device) receives the number of waits that ran out.
 * d_scratch: device, 256 + 8 n bytes rounded up to a multiple of 256
 * (lu_refine_workspace_size(n) bytes suffice). */
LU_API lu_status lu_selftest_wait_solve_c(lu_stream_t stream, unsigned long long wait_ns,
                                          int64_t n, const float* d_lu, int64_t ldlu,
                                          double* d_x, void* d_scratch, size_t bytes,
                                          unsigned* d_expired);

/* One block row of the host entry's left-looking chunk catch-up, for tests
 * and measurement (no reference counterpart; for one block row it stands
 * for the U-panel solves of src/lu_nopiv_inner_rl.hxx:155-190 that the
 * reference runs per outer step).  d_a holds, column-major with leading
 * dimension lda, a factored in x in diagonal block at (0, 0) (its unit
 * lower part is used) and the block row R (in x nc) at column coff >= in.
 * First R loses the sum of nslabs fp32 slabs of partial products (slab s,
 * column q, row i at d_part[s * slab + q * ldp + i], ldp = in rounded up to
 * a multiple of 4, slab a multiple of 4; summed in slab order, then one
 * subtraction, as the split-K finish does; nslabs = 0: none).  Then R -= La
 * Xb with K = kl (kl = 0: nothing; fp16 operands, bf16 if bf16 != 0; La row
 * i at d_la + i * lda_k elements, Xb column q at d_xb + q * ldx), then R =
 * L^{-1} R in place, and R's fp16 / bf16 copy to d_xo (column q at d_xo + q
 * * ldx).  fused = 1: one launch (in and kl multiples of 32, in <= 256, ldx
 * and lda_k multiples of 8, operand pointers 16-byte aligned); fused = 0:
 * the split-K finish, the tensor-core update and the blocked U-panel
 * solves.  Everything but the order of the sum La Xb is the same bit for
 * bit either way.  d_err: device int, the update's error word (0 on
 * success). */
LU_API lu_status lu_catchup_row_step_c(lu_stream_t stream, int fused, int bf16, int64_t in,
                                       int64_t nc, int64_t coff, int64_t kl, float* d_a,
                                       int64_t lda, const void* d_la, int64_t lda_k,
                                       const void* d_xb, void* d_xo, int64_t ldx,
                                       const float* d_part, int64_t slab, int64_t ldp,
                                       int nslabs, int* d_err);

/* ---- profiling (new; the reference only wall-clocks whole calls) ------- */
typedef struct lu_profile_entry {
  char name[32];     /* kernel class, e.g. "tc_update", "diag_factor" */
  int64_t launches;  /* launches recorded */
  double total_ms;   /* summed CUDA-event time on the launching stream */
  double bytes;      /* summed algorithmic bytes (HBM-bound kernels) */
  double flops;      /* summed algorithmic flops */
} lu_profile_entry;

/* Start recording CUDA events around each kernel class (clears old data). */
LU_API void lu_profile_begin(void);
/* Stop recording, wait for the recorded events and write up to max_entries
 * aggregated entries; returns the number of kernel classes seen. */
LU_API int lu_profile_end(lu_profile_entry* out, int max_entries);
/* Per-launch timeline of the last profiled region (after lu_profile_end):
 * kernel class, stream (numbered in order of first use) and start / end in
 * ms from the first recorded launch.  Returns the number of launches. */
typedef struct lu_trace_entry {
  char name[32];
  int32_t stream;
  double start_ms, end_ms;
} lu_trace_entry;
LU_API int lu_profile_trace(lu_trace_entry* out, int max_entries);
/* Number of kernels this library has launched in this process. */
LU_API long long lu_launch_count(void);

/* Device memory the library allocates for itself (a workspace not supplied
 * by the caller, the host entry's operand buffers, solve scratch) comes from
 * a stream-ordered memory pool per device that keeps freed blocks for the
 * next call.  lu_trim_memory_c synchronises the current device and returns
 * the pool's unused memory to the driver (no reference counterpart). */
LU_API lu_status lu_trim_memory_c(void);

#ifdef __cplusplus
}
#endif
#endif /* LU_B200_H */
