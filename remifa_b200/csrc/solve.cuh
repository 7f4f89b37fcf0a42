// Triangular solves and FP64 residuals (solve.cu).
#pragma once

#include "common.cuh"

namespace lub {

// op(T) X = X in place, T = the unit-lower L (upper = false) or the upper U
// (upper = true) of the in-place factors lu (fp32, ld); op = T or T^T;
// X fp64 n x nrhs (ldx).  One solve launch per triangle (plus a copy kernel
// that moves X into B, n x nrhs with ld n, for groups of 1-2 columns).
// sync: trsm_sync_bytes(nrhs) bytes of device memory.  sync and B are not
// shared with a solve in flight on another stream.  trsm_ws_bytes = both.
size_t trsm_sync_bytes(int64_t nrhs);
size_t trsm_ws_bytes(int64_t n, int64_t nrhs);
// wait_ns / withhold: the self-test of the give-up path only (a bound of
// wait_ns per wait instead of 4 s; the block solved first does not publish,
// so the waits for it run out and the solve ends with NaN).
lu_status launch_trsm(cudaStream_t st, int64_t n, const float* lu, int64_t ld,
                      double* X, int64_t ldx, int64_t nrhs, bool upper,
                      bool trans, unsigned* sync, double* B,
                      unsigned long long wait_ns = 0, int withhold = -1);
// X <- (L U)^-1 X (trans: (L U)^-T X): two launch_trsm.
lu_status launch_lu_solve(cudaStream_t st, int64_t n, const float* lu, int64_t ld,
                          double* X, int64_t ldx, int64_t nrhs, bool trans, unsigned* sync,
                          double* B);

// Workspace (bytes) of launch_residual / launch_norm_inf for size n.
size_t residual_ws_bytes(int64_t n);

// r = b - A x (fp64, deterministic order); maxes[0..2] receive the bit
// patterns of max|r|, max|x|, max|b|.
lu_status launch_residual(cudaStream_t st, int64_t n, const float* A,
                          int64_t lda, const double* b, const double* x,
                          double* r, void* ws, unsigned long long* maxes);

// *out = bit pattern of ||A||_inf (max row sum of |a_ij|).
lu_status launch_norm_inf(cudaStream_t st, int64_t n, const float* A,
                          int64_t lda, void* ws, unsigned long long* out);

// R = B - op(A) X for nrhs >= 1 columns at once (A read once per group of 8
// columns; fp64, fixed summation order); maxes[3c .. 3c+2] receive the bit
// patterns of max|r|, max|x|, max|b| of column c.
lu_status launch_residual_multi(cudaStream_t st, int64_t n, int64_t nrhs, const float* A,
                                int64_t lda, const double* B, int64_t ldb, const double* X,
                                int64_t ldx, double* R, int64_t ldr, bool trans,
                                unsigned long long* maxes);

// x += d
lu_status launch_axpy(cudaStream_t st, int64_t n, const double* d, double* x);

// adjoint.cu: dA = alpha * P Q^T (fp64 in, fp32 out); r = b - A^T x; ||A||_1
lu_status launch_outer(cudaStream_t st, int64_t n, int64_t k, double alpha,
                       const double* P, int64_t ldp, const double* Q, int64_t ldq,
                       float* dA, int64_t ldda);
lu_status launch_residual_t(cudaStream_t st, int64_t n, const float* A,
                            int64_t lda, const double* b, const double* x,
                            double* r, unsigned long long* maxes);
lu_status launch_norm_one(cudaStream_t st, int64_t n, const float* A,
                          int64_t lda, unsigned long long* out);

// refine.cu: the host-side argument checks of lu_refine_ex_c (sizes, leading
// dimensions, tol, max_iter, trans, and non-null pointers when there is work)
// and its device check (an sm_100 device current).  Neither touches the
// device's memory or loads a module.
lu_status refine_check_args(int64_t n, int64_t nrhs, const float* d_a, int64_t lda,
                            const float* d_lu, int64_t ldlu, const double* d_b,
                            int64_t ldb, const double* d_x, int64_t ldx, int trans,
                            double tol, int max_iter);
lu_status refine_check_device();

}  // namespace lub
