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

#include <cmath>
#include <cstring>

using namespace lub;

namespace {

struct RefineWs {
  size_t off_r, off_d, off_p, off_max, bytes;
};

RefineWs refine_layout(int64_t n) {
  RefineWs w;
  size_t off = 0;
  w.off_r = off; off = align_up(off + (size_t)n * 8, 256);
  w.off_d = off; off = align_up(off + (size_t)n * 8, 256);
  w.off_p = off; off = align_up(off + residual_ws_bytes(n), 256);
  w.off_max = off; off += 256;
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
  if (!trans) {  // L U x = b: L y = b, then U x = y
    LUB_TRY(launch_trsm(st, n, d_lu, ldlu, d_x, ldx, nrhs, false, false));
    return launch_trsm(st, n, d_lu, ldlu, d_x, ldx, nrhs, true, false);
  }
  // (L U)^T x = U^T L^T x = b: U^T y = b, then L^T x = y
  LUB_TRY(launch_trsm(st, n, d_lu, ldlu, d_x, ldx, nrhs, true, true));
  return launch_trsm(st, n, d_lu, ldlu, d_x, ldx, nrhs, false, true);
}

LU_API lu_status lu_refine_workspace_size(int64_t n, size_t* bytes) {
  if (n < 0 || !bytes) return LU_ERR_INVALID_ARG;
  *bytes = refine_layout(n).bytes;
  return LU_SUCCESS;
}

}  // extern "C"

namespace {

// One right-hand side; trans: refine A^T x = b.
lu_status refine_one(lu_stream_t stream, int64_t n, const float* d_a,
                     int64_t lda, const float* d_lu, int64_t ldlu,
                     const double* d_b, double* d_x, int trans, double tol,
                     int max_iter, char* wb, const RefineWs& w, int* iters,
                     double* berr) {
  cudaStream_t st = (cudaStream_t)stream;
  double* r = reinterpret_cast<double*>(wb + w.off_r);
  double* d = reinterpret_cast<double*>(wb + w.off_d);
  void* P = wb + w.off_p;
  unsigned long long* mx = reinterpret_cast<unsigned long long*>(wb + w.off_max);
  lu_status s = LU_SUCCESS;
  double e = INFINITY;
  int it = 0;
  unsigned long long h[4] = {0, 0, 0, 0};
  do {
    s = trans ? launch_norm_one(st, n, d_a, lda, mx + 3)
              : launch_norm_inf(st, n, d_a, lda, P, mx + 3);
    if (s != LU_SUCCESS) break;
    if (cudaMemcpyAsync(d_x, d_b, (size_t)n * 8, cudaMemcpyDeviceToDevice, st) != cudaSuccess) {
      s = LU_ERR_CUDA;
      break;
    }
    if ((s = lu_solve_c(stream, n, d_lu, ldlu, d_x, n, 1, trans)) != LU_SUCCESS) break;
    for (;;) {
      s = trans ? launch_residual_t(st, n, d_a, lda, d_b, d_x, r, mx)
                : launch_residual(st, n, d_a, lda, d_b, d_x, r, P, mx);
      if (s != LU_SUCCESS) break;
      if (cudaMemcpyAsync(h, mx, sizeof(h), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
          cudaStreamSynchronize(st) != cudaSuccess) {
        s = LU_ERR_CUDA;
        break;
      }
      const double rmax = bits_to_double(h[0]), xmax = bits_to_double(h[1]);
      const double bmax = bits_to_double(h[2]), anorm = bits_to_double(h[3]);
      const double den = anorm * xmax + bmax;
      e = den > 0.0 ? rmax / den : (rmax > 0.0 ? INFINITY : 0.0);
      if (std::isnan(e)) break;
      if (e <= tol || it >= max_iter) break;
      if (cudaMemcpyAsync(d, r, (size_t)n * 8, cudaMemcpyDeviceToDevice, st) != cudaSuccess) {
        s = LU_ERR_CUDA;
        break;
      }
      if ((s = lu_solve_c(stream, n, d_lu, ldlu, d, n, 1, trans)) != LU_SUCCESS) break;
      if ((s = launch_axpy(st, n, d, d_x)) != LU_SUCCESS) break;
      ++it;
    }
  } while (false);
  if (iters) *iters = it;
  if (berr) *berr = e;
  return s;
}

}  // namespace

extern "C" {

LU_API lu_status lu_refine_ex_c(lu_stream_t stream, int64_t n, int64_t nrhs,
                                const float* d_a, int64_t lda, const float* d_lu,
                                int64_t ldlu, const double* d_b, int64_t ldb,
                                double* d_x, int64_t ldx, int trans, double tol,
                                int max_iter, int* iters, double* berr,
                                void* workspace, size_t ws_bytes) {
  if (n < 0 || nrhs < 0 || lda < std::max<int64_t>(1, n) ||
      ldlu < std::max<int64_t>(1, n) || ldb < std::max<int64_t>(1, n) ||
      ldx < std::max<int64_t>(1, n) || max_iter < 0 || !(tol >= 0.0) ||
      (trans != 0 && trans != 1))
    return LU_ERR_INVALID_ARG;
  if (iters) *iters = 0;
  if (berr) *berr = 0.0;
  if (n == 0 || nrhs == 0) return LU_SUCCESS;
  if (!d_a || !d_lu || !d_b || !d_x) return LU_ERR_INVALID_ARG;
  LUB_TRY(check_device_local());
  const RefineWs w = refine_layout(n);
  if (workspace && ws_bytes < w.bytes) return LU_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  void* ws = workspace;
  bool owned = false;
  if (!ws) {
    if (cudaMallocAsync(&ws, w.bytes, st) != cudaSuccess) return LU_ERR_ALLOC;
    owned = true;
  }
  lu_status s = LU_SUCCESS;
  int it_max = 0;
  double e_max = 0.0;
  for (int64_t c = 0; c < nrhs && s == LU_SUCCESS; ++c) {
    int it = 0;
    double e = 0.0;
    s = refine_one(stream, n, d_a, lda, d_lu, ldlu, d_b + c * ldb, d_x + c * ldx,
                   trans, tol, max_iter, static_cast<char*>(ws), w, &it, &e);
    it_max = std::max(it_max, it);
    e_max = std::isnan(e) ? e : std::max(e_max, e);
  }
  if (owned) cudaFreeAsync(ws, st);
  if (iters) *iters = it_max;
  if (berr) *berr = e_max;
  if (s == LU_SUCCESS && !(e_max <= tol)) s = LU_ERR_NOT_CONVERGED;
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
