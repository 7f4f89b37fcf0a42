// Solve and FP64 iterative refinement entry points (host drivers).
//
// New relative to the reference, whose harness solves on the host in the
// working precision (tests/testing_lu_gpu.hxx:1309-1313): refinement reaches
// an fp64-level backward error from a factorization whose trailing updates
// ran in fp16 / bf16 / e4m3 on the tensor cores.
//   x0 = U^-1 L^-1 b                  (fp32 factors, fp64 arithmetic)
//   repeat: r = b - A x   (fp64, A the original fp32 matrix)
//           berr = ||r||_inf / (||A||_inf ||x||_inf + ||b||_inf)
//           stop when berr <= tol;  x += U^-1 L^-1 r
#include "common.cuh"
#include "kernels.cuh"
#include "solve.cuh"
#include "lu_b200.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

using namespace lub;

namespace {

struct RefineWs {
  size_t off_r, off_d, off_p, off_max, off_sync, bytes;
};

// Residuals and corrections of all nrhs columns, one set of chunk partial
// sums (the columns' residuals run one after another), and per column the
// three maxima of the backward error plus the matrix norm; the counters of
// the triangular solves.
RefineWs refine_layout(int64_t n, int64_t nrhs = 1) {
  RefineWs w;
  size_t off = 0;
  w.off_r = off; off = align_up(off + (size_t)n * nrhs * 8, 256);
  w.off_d = off; off = align_up(off + (size_t)n * nrhs * 8, 256);
  w.off_p = off; off = align_up(off + residual_ws_bytes(n), 256);
  w.off_max = off; off = align_up(off + (size_t)(3 * nrhs + 1) * 8, 256);
  w.off_sync = off; off = align_up(off + trsm_sync_bytes(nrhs), 256);
  w.bytes = off;
  return w;
}

double bits_to_double(unsigned long long b) {
  double d;
  std::memcpy(&d, &b, sizeof(d));
  return d;
}

lu_status check_device_local() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return LU_ERR_NO_DEVICE;
  int major = 0;
  if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev) != cudaSuccess)
    return LU_ERR_NO_DEVICE;
  return major == 10 ? LU_SUCCESS : LU_ERR_NO_DEVICE;
}

}  // namespace

extern "C" {

LU_API lu_status lu_solve_c(lu_stream_t stream, int64_t n, const float* d_lu,
                            int64_t ldlu, double* d_x, int64_t ldx,
                            int64_t nrhs, int trans) {
  if (n < 0 || nrhs < 0 || ldlu < std::max<int64_t>(1, n) ||
      ldx < std::max<int64_t>(1, n) || (trans != 0 && trans != 1))
    return LU_ERR_INVALID_ARG;
  if (n == 0 || nrhs == 0) return LU_SUCCESS;
  if (!d_lu || !d_x) return LU_ERR_INVALID_ARG;
  LUB_TRY(check_device_local());
  cudaStream_t st = (cudaStream_t)stream;
  // the solve's counter words and right-hand-side copy come from the
  // stream-ordered allocator
  void* ws = nullptr;
  if (pool_malloc_async((void**)&ws, trsm_ws_bytes(n, nrhs), st) != cudaSuccess) return LU_ERR_ALLOC;
  const lu_status s = launch_lu_solve(
      st, n, d_lu, ldlu, d_x, ldx, nrhs, trans != 0, static_cast<unsigned*>(ws),
      reinterpret_cast<double*>(static_cast<char*>(ws) + trsm_sync_bytes(nrhs)));
  cudaFreeAsync(ws, st);
  return s;
}

LU_API lu_status lu_refine_workspace_size(int64_t n, size_t* bytes) {
  if (n < 0 || !bytes) return LU_ERR_INVALID_ARG;
  *bytes = refine_layout(n).bytes;
  return LU_SUCCESS;
}

}  // extern "C"

namespace {

// All nrhs columns together; trans: refine A^T X = B.  Per iteration: the
// fp64 residual of every column, one read-back of all backward errors, then
// one multi-column triangular solve of the corrections.
lu_status refine_multi(lu_stream_t stream, int64_t n, int64_t nrhs, const float* d_a,
                       int64_t lda, const float* d_lu, int64_t ldlu, const double* d_b,
                       int64_t ldb, double* d_x, int64_t ldx, int trans, double tol,
                       int max_iter, char* wb, const RefineWs& w, int* iters,
                       double* berr) {
  cudaStream_t st = (cudaStream_t)stream;
  double* R = reinterpret_cast<double*>(wb + w.off_r);
  double* D = reinterpret_cast<double*>(wb + w.off_d);
  void* P = wb + w.off_p;
  unsigned long long* mx = reinterpret_cast<unsigned long long*>(wb + w.off_max);
  unsigned long long* mnorm = mx + 3 * nrhs;
  std::vector<unsigned long long> h((size_t)(3 * nrhs + 1));
  double e = INFINITY;
  int it = 0;
  LUB_TRY(trans ? launch_norm_one(st, n, d_a, lda, mnorm)
                : launch_norm_inf(st, n, d_a, lda, P, mnorm));
  LUB_CUDA_TRY(cudaMemcpy2DAsync(d_x, (size_t)ldx * 8, d_b, (size_t)ldb * 8, (size_t)n * 8,
                                 (size_t)nrhs, cudaMemcpyDeviceToDevice, st));
  // the solves copy their right-hand sides into R (free until the next
  // residual) and count tickets in the sync words
  unsigned* sync = reinterpret_cast<unsigned*>(wb + w.off_sync);
  LUB_TRY(launch_lu_solve(st, n, d_lu, ldlu, d_x, ldx, nrhs, trans != 0, sync, R));
  for (;;) {
    if (nrhs > 1) {
      // all columns in one pass over A
      LUB_TRY(launch_residual_multi(st, n, nrhs, d_a, lda, d_b, ldb, d_x, ldx, R, n,
                                    trans != 0, mx));
    } else {
      LUB_TRY(trans ? launch_residual_t(st, n, d_a, lda, d_b, d_x, R, mx)
                    : launch_residual(st, n, d_a, lda, d_b, d_x, R, P, mx));
    }
    LUB_CUDA_TRY(cudaMemcpyAsync(h.data(), mx, h.size() * 8, cudaMemcpyDeviceToHost, st));
    LUB_CUDA_TRY(cudaStreamSynchronize(st));
    const double anorm = bits_to_double(h[3 * nrhs]);
    e = 0.0;
    for (int64_t c = 0; c < nrhs; ++c) {
      const double rmax = bits_to_double(h[3 * c]), xmax = bits_to_double(h[3 * c + 1]);
      const double bmax = bits_to_double(h[3 * c + 2]);
      const double den = anorm * xmax + bmax;
      const double ec = den > 0.0 ? rmax / den : (rmax > 0.0 ? INFINITY : 0.0);
      if (std::isnan(ec)) {
        e = ec;
        break;
      }
      e = std::max(e, ec);
    }
    if (std::isnan(e) || e <= tol || it >= max_iter) break;
    LUB_CUDA_TRY(cudaMemcpyAsync(D, R, (size_t)n * nrhs * 8, cudaMemcpyDeviceToDevice, st));
    LUB_TRY(launch_lu_solve(st, n, d_lu, ldlu, D, n, nrhs, trans != 0, sync, R));
    for (int64_t c = 0; c < nrhs; ++c) LUB_TRY(launch_axpy(st, n, D + c * n, d_x + c * ldx));
    ++it;
  }
  if (iters) *iters = it;
  if (berr) *berr = e;
  return LU_SUCCESS;
}

}  // namespace

namespace lub {

lu_status refine_check_args(int64_t n, int64_t nrhs, const float* d_a, int64_t lda,
                            const float* d_lu, int64_t ldlu, const double* d_b,
                            int64_t ldb, const double* d_x, int64_t ldx, int trans,
                            double tol, int max_iter) {
  if (n < 0 || nrhs < 0 || lda < std::max<int64_t>(1, n) ||
      ldlu < std::max<int64_t>(1, n) || ldb < std::max<int64_t>(1, n) ||
      ldx < std::max<int64_t>(1, n) || max_iter < 0 || !(tol >= 0.0) ||
      (trans != 0 && trans != 1))
    return LU_ERR_INVALID_ARG;
  if (n > 0 && nrhs > 0 && (!d_a || !d_lu || !d_b || !d_x)) return LU_ERR_INVALID_ARG;
  return LU_SUCCESS;
}

lu_status refine_check_device() { return check_device_local(); }

}  // namespace lub

extern "C" {

LU_API lu_status lu_refine_ex_workspace_size(int64_t n, int64_t nrhs, size_t* bytes) {
  if (n < 0 || nrhs < 0 || !bytes) return LU_ERR_INVALID_ARG;
  *bytes = refine_layout(n, std::max<int64_t>(nrhs, 1)).bytes;
  return LU_SUCCESS;
}

LU_API lu_status lu_refine_ex_c(lu_stream_t stream, int64_t n, int64_t nrhs,
                                const float* d_a, int64_t lda, const float* d_lu,
                                int64_t ldlu, const double* d_b, int64_t ldb,
                                double* d_x, int64_t ldx, int trans, double tol,
                                int max_iter, int* iters, double* berr,
                                void* workspace, size_t ws_bytes) {
  LUB_TRY(refine_check_args(n, nrhs, d_a, lda, d_lu, ldlu, d_b, ldb, d_x, ldx, trans,
                            tol, max_iter));
  if (iters) *iters = 0;
  if (berr) *berr = 0.0;
  if (n == 0 || nrhs == 0) return LU_SUCCESS;
  LUB_TRY(check_device_local());
  const RefineWs w = refine_layout(n, nrhs);
  if (workspace && ws_bytes < w.bytes) return LU_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  void* ws = workspace;
  bool owned = false;
  if (!ws) {
    if (pool_malloc_async((void**)&ws, w.bytes, st) != cudaSuccess) return LU_ERR_ALLOC;
    owned = true;
  }
  double e = 0.0;
  const lu_status s = refine_multi(stream, n, nrhs, d_a, lda, d_lu, ldlu, d_b, ldb, d_x,
                                   ldx, trans, tol, max_iter, static_cast<char*>(ws), w,
                                   iters, &e);
  if (owned) cudaFreeAsync(ws, st);
  if (berr) *berr = e;
  if (s == LU_SUCCESS && !(e <= tol)) return LU_ERR_NOT_CONVERGED;
  return s;
}

LU_API lu_status lu_refine_c(lu_stream_t stream, int64_t n, const float* d_a,
                             int64_t lda, const float* d_lu, int64_t ldlu,
                             const double* d_b, double* d_x, double tol,
                             int max_iter, int* iters, double* berr,
                             void* workspace, size_t ws_bytes) {
  return lu_refine_ex_c(stream, n, 1, d_a, lda, d_lu, ldlu, d_b,
                        std::max<int64_t>(1, n), d_x, std::max<int64_t>(1, n), 0,
                        tol, max_iter, iters, berr, workspace, ws_bytes);
}

}  // extern "C"
