// GMRES-based iterative refinement (new; the reference has no refinement).
//
// Classic refinement (refine.cu) corrects x with (LU)^-1 r; it converges
// while kappa(A) times the factorization's relative error stays below one,
// which fails for low-precision factors of ill-conditioned matrices (an
// fp16 / bf16 / e4m3 Schur update at kappa ~ 1e4 .. 1e6).  GMRES-IR (Carson
// and Higham, SIAM J. Sci. Comput. 40(2), 2018) instead solves each
// correction equation A d = r by GMRES on the preconditioned system
// (LU)^-1 A d = (LU)^-1 r, all in fp64, so the low-precision factors only
// need to make (LU)^-1 A well enough conditioned for GMRES:
//
//   x = (LU)^-1 b
//   repeat: r = b - A x (fp64), stop when the normwise backward error
//           ||r||inf / (||A||inf ||x||inf + ||b||inf) <= tol
//           z = (LU)^-1 r, beta = ||z||, v0 = z / beta
//           Arnoldi on M = (LU)^-1 A (classical Gram-Schmidt applied twice,
//           one read-back of the new Hessenberg column per step), Givens
//           rotations on the host, until |g_{j+1}| <= inner_tol beta or the
//           restart length m; x += V y with H y = g.
//
// Device work per Arnoldi step: one fp64 product with the fp32 A (its
// deterministic chunked sums, launch_residual with b = 0), the two
// triangular solves, two passes of V^T w / w - V h and a norm, each a fixed
// reduction order so a run is reproducible bit for bit.
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

constexpr int kDotT = 1024;  // threads of the single-CTA reductions

// out[c] = sum_i V[i + c n] w[i] for c < k (one CTA per column; each thread
// sums its strided rows in order, then a fixed tree).
__global__ void __launch_bounds__(kDotT)
dots_kernel(int64_t n, int k, const double* __restrict__ V, const double* __restrict__ w,
            double* __restrict__ out) {
  __shared__ double red[kDotT];
  const int c = blockIdx.x;
  if (c >= k) return;
  const double* v = V + (int64_t)c * n;
  double s = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += kDotT) s = fma(v[i], w[i], s);
  red[threadIdx.x] = s;
  __syncthreads();
  for (int h = kDotT / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[c] = red[0];
}

// w[i] -= sum_{c<k} V[i + c n] h[c]  (sign = -1), or x[i] += ... (sign = +1).
__global__ void gemv_kernel(int64_t n, int k, const double* __restrict__ V,
                            const double* __restrict__ h, double sign,
                            double* __restrict__ w) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double s = 0.0;
  for (int c = 0; c < k; ++c) s = fma(V[i + (int64_t)c * n], h[c], s);
  w[i] = fma(sign, s, w[i]);
}

// h[c] += g[c] for c < k (the second Gram-Schmidt pass's coefficients).
__global__ void add_kernel(int k, const double* __restrict__ g, double* __restrict__ h) {
  const int c = threadIdx.x;
  if (c < k) h[c] += g[c];
}

// out = ||w||^2 (one CTA, fixed order).
__global__ void __launch_bounds__(kDotT)
nrm2sq_kernel(int64_t n, const double* __restrict__ w, double* __restrict__ out) {
  __shared__ double red[kDotT];
  double s = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += kDotT) s = fma(w[i], w[i], s);
  red[threadIdx.x] = s;
  __syncthreads();
  for (int h = kDotT / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = red[0];
}

// y = s * x
__global__ void scale_kernel(int64_t n, double s, const double* __restrict__ x,
                             double* __restrict__ y) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] = s * x[i];
}

unsigned grid_of(int64_t n) { return (unsigned)ceil_div(n, 256); }

struct GmresWs {
  size_t off_v, off_w, off_r, off_z, off_b0, off_p, off_max, off_h, off_g, off_sync,
      off_tb, bytes;
};

GmresWs gmres_layout(int64_t n, int m) {
  GmresWs w;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t o = off;
    off = align_up(off + bytes, 256);
    return o;
  };
  w.off_v = take((size_t)n * (m + 1) * 8);   // Krylov basis
  w.off_w = take((size_t)n * 8);             // new Arnoldi vector
  w.off_r = take((size_t)n * 8);             // residual
  w.off_z = take((size_t)n * 8);             // spare vector
  w.off_b0 = take((size_t)n * 8);            // zeros: -A v = 0 - A v
  w.off_p = take(residual_ws_bytes(n));      // chunk partial sums
  w.off_max = take(8 * 8);                   // backward-error maxima, ||A||
  w.off_h = take((size_t)(m + 2) * 8);       // Hessenberg column (+ norm^2)
  w.off_g = take((size_t)(m + 2) * 8);       // second-pass coefficients
  w.off_sync = take(trsm_ws_bytes(n, 1));    // triangular solves
  w.off_tb = 0;
  w.bytes = off;
  return w;
}

double bits_d(unsigned long long b) {
  double d;
  std::memcpy(&d, &b, sizeof(d));
  return d;
}

}  // namespace

extern "C" {

LU_API lu_status lu_gmres_ir_workspace_size(int64_t n, int restart, size_t* bytes) {
  if (n < 0 || restart < 1 || restart > LU_GMRES_MAX_RESTART || !bytes)
    return LU_ERR_INVALID_ARG;
  *bytes = gmres_layout(n, restart).bytes;
  return LU_SUCCESS;
}

LU_API lu_status lu_gmres_ir_c(lu_stream_t stream, int64_t n, const float* d_a, int64_t lda,
                               const float* d_lu, int64_t ldlu, const double* d_b,
                               double* d_x, double tol, int max_outer, int restart,
                               double inner_tol, int* outer_iters, int* inner_iters,
                               double* berr, void* workspace, size_t ws_bytes) {
  const int64_t one = std::max<int64_t>(1, n);
  LUB_TRY(refine_check_args(n, 1, d_a, lda, d_lu, ldlu, d_b, one, d_x, one, 0, tol,
                            max_outer));
  if (restart < 1 || restart > LU_GMRES_MAX_RESTART || !(inner_tol > 0.0) || inner_tol >= 1.0)
    return LU_ERR_INVALID_ARG;
  if (outer_iters) *outer_iters = 0;
  if (inner_iters) *inner_iters = 0;
  if (berr) *berr = 0.0;
  if (n == 0) return LU_SUCCESS;
  LUB_TRY(refine_check_device());
  const int m = restart;
  const GmresWs L = gmres_layout(n, m);
  if (workspace && ws_bytes < L.bytes) return LU_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  void* ws = workspace;
  bool owned = false;
  if (!ws) {
    if (pool_malloc_async((void**)&ws, L.bytes, st) != cudaSuccess) return LU_ERR_ALLOC;
    owned = true;
  }
  char* wb = static_cast<char*>(ws);
  double* V = reinterpret_cast<double*>(wb + L.off_v);
  double* w = reinterpret_cast<double*>(wb + L.off_w);
  double* r = reinterpret_cast<double*>(wb + L.off_r);
  double* zero = reinterpret_cast<double*>(wb + L.off_b0);
  void* P = wb + L.off_p;
  unsigned long long* mx = reinterpret_cast<unsigned long long*>(wb + L.off_max);
  double* h = reinterpret_cast<double*>(wb + L.off_h);
  double* g2 = reinterpret_cast<double*>(wb + L.off_g);
  unsigned* sync = reinterpret_cast<unsigned*>(wb + L.off_sync);
  double* tb = reinterpret_cast<double*>(wb + L.off_sync + trsm_sync_bytes(1));

  lu_status s = LU_SUCCESS;
  int outer = 0, inner_total = 0;
  double e = INFINITY;
  // H column-major (m + 1) x m on the host, Givens cosines / sines, g
  std::vector<double> H((size_t)(m + 1) * m), cs(m), sn(m), gv(m + 1), y(m), hcol(m + 2);
  auto run = [&]() -> lu_status {
    LUB_CUDA_TRY(cudaMemsetAsync(zero, 0, (size_t)n * 8, st));
    LUB_TRY(launch_norm_inf(st, n, d_a, lda, P, mx + 3));
    LUB_CUDA_TRY(cudaMemcpyAsync(d_x, d_b, (size_t)n * 8, cudaMemcpyDeviceToDevice, st));
    LUB_TRY(launch_lu_solve(st, n, d_lu, ldlu, d_x, n, 1, false, sync, tb));
    for (;;) {
      // r = b - A x and the backward error
      LUB_TRY(launch_residual(st, n, d_a, lda, d_b, d_x, r, P, mx));
      unsigned long long hm[4];
      LUB_CUDA_TRY(cudaMemcpyAsync(hm, mx, sizeof(hm), cudaMemcpyDeviceToHost, st));
      LUB_CUDA_TRY(cudaStreamSynchronize(st));
      const double den = bits_d(hm[3]) * bits_d(hm[1]) + bits_d(hm[2]);
      e = den > 0.0 ? bits_d(hm[0]) / den : (bits_d(hm[0]) > 0.0 ? INFINITY : 0.0);
      if (std::isnan(e) || e <= tol || outer >= max_outer) return LU_SUCCESS;
      // z = (LU)^-1 r, beta = ||z||, v0 = z / beta
      LUB_CUDA_TRY(cudaMemcpyAsync(w, r, (size_t)n * 8, cudaMemcpyDeviceToDevice, st));
      LUB_TRY(launch_lu_solve(st, n, d_lu, ldlu, w, n, 1, false, sync, tb));
      nrm2sq_kernel<<<1, kDotT, 0, st>>>(n, w, h);
      LUB_LAUNCH_CHECK();
      double beta2 = 0.0;
      LUB_CUDA_TRY(cudaMemcpyAsync(&beta2, h, 8, cudaMemcpyDeviceToHost, st));
      LUB_CUDA_TRY(cudaStreamSynchronize(st));
      const double beta = std::sqrt(beta2);
      if (!(beta > 0.0) || !std::isfinite(beta)) {
        e = std::isfinite(beta) ? e : NAN;
        return LU_SUCCESS;
      }
      scale_kernel<<<grid_of(n), 256, 0, st>>>(n, 1.0 / beta, w, V);
      LUB_LAUNCH_CHECK();
      std::fill(gv.begin(), gv.end(), 0.0);
      gv[0] = beta;
      int k = 0;  // Arnoldi steps taken
      for (int j = 0; j < m; ++j) {
        double* vj = V + (int64_t)j * n;
        // w = (LU)^-1 (A v_j): the residual kernel gives 0 - A v_j
        LUB_TRY(launch_residual(st, n, d_a, lda, zero, vj, w, P, mx));
        LUB_TRY(launch_lu_solve(st, n, d_lu, ldlu, w, n, 1, false, sync, tb));
        // classical Gram-Schmidt twice against v_0 .. v_j (w holds -M v_j)
        dots_kernel<<<j + 1, kDotT, 0, st>>>(n, j + 1, V, w, h);
        gemv_kernel<<<grid_of(n), 256, 0, st>>>(n, j + 1, V, h, -1.0, w);
        dots_kernel<<<j + 1, kDotT, 0, st>>>(n, j + 1, V, w, g2);
        gemv_kernel<<<grid_of(n), 256, 0, st>>>(n, j + 1, V, g2, -1.0, w);
        add_kernel<<<1, 64, 0, st>>>(j + 1, g2, h);
        nrm2sq_kernel<<<1, kDotT, 0, st>>>(n, w, h + j + 1);
        LUB_LAUNCH_CHECK();
        LUB_CUDA_TRY(cudaMemcpyAsync(hcol.data(), h, (size_t)(j + 2) * 8,
                                     cudaMemcpyDeviceToHost, st));
        LUB_CUDA_TRY(cudaStreamSynchronize(st));
        ++k;
        ++inner_total;
        // the column of M v_j: negate (w held -M v_j)
        double* col = H.data() + (size_t)j * (m + 1);
        for (int i = 0; i <= j; ++i) col[i] = -hcol[i];
        const double hn = std::sqrt(hcol[j + 1]);
        col[j + 1] = hn;
        // v_{j+1} = -w / hn  (= (M v_j - sum h_i v_i) / hn)
        if (hn > 0.0 && j + 1 <= m)
          scale_kernel<<<grid_of(n), 256, 0, st>>>(n, -1.0 / hn, w, V + (int64_t)(j + 1) * n);
        LUB_LAUNCH_CHECK();
        // Givens rotations: apply the previous ones, make a new one
        for (int i = 0; i < j; ++i) {
          const double t = cs[i] * col[i] + sn[i] * col[i + 1];
          col[i + 1] = -sn[i] * col[i] + cs[i] * col[i + 1];
          col[i] = t;
        }
        const double rr = std::hypot(col[j], col[j + 1]);
        cs[j] = rr > 0.0 ? col[j] / rr : 1.0;
        sn[j] = rr > 0.0 ? col[j + 1] / rr : 0.0;
        col[j] = rr;
        col[j + 1] = 0.0;
        gv[j + 1] = -sn[j] * gv[j];
        gv[j] = cs[j] * gv[j];
        if (!(hn > 0.0) || std::fabs(gv[j + 1]) <= inner_tol * beta) break;
      }
      // H(0:k, 0:k) y = g(0:k), back substitution; x += V y
      for (int i = k - 1; i >= 0; --i) {
        double t = gv[i];
        for (int c = i + 1; c < k; ++c) t -= H[(size_t)c * (m + 1) + i] * y[c];
        y[i] = t / H[(size_t)i * (m + 1) + i];
      }
      LUB_CUDA_TRY(cudaMemcpyAsync(g2, y.data(), (size_t)k * 8, cudaMemcpyHostToDevice, st));
      gemv_kernel<<<grid_of(n), 256, 0, st>>>(n, k, V, g2, 1.0, d_x);
      LUB_LAUNCH_CHECK();
      ++outer;
    }
  };
  s = run();
  if (owned) cudaFreeAsync(ws, st);
  if (outer_iters) *outer_iters = outer;
  if (inner_iters) *inner_iters = inner_total;
  if (berr) *berr = e;
  if (s == LU_SUCCESS && !(e <= tol)) return LU_ERR_NOT_CONVERGED;
  return s;
}

}  // extern "C"
