// Adjoint of the LU solve X = A^-1 B (new; the reference has no derivative).
//
// For a loss L(X):  dL/dB = A^-T G  and  dL/dA = -(A^-T G) X^T,  G = dL/dX.
// Both reuse the forward factors: A^-T G is two transposed triangular solves
// (U^T then L^T, solve.cu), and dA is one rank-nrhs outer product computed
// here in fp64 and stored in fp32.  Also: transposed FP64 residuals so the
// adjoint system can be refined like the forward one.
#include "common.cuh"
#include "kernels.cuh"
#include "solve.cuh"
#include "lu_b200.h"

#include <algorithm>

namespace lub {
namespace {

constexpr int OT = 64;   // dA tile
constexpr int OR = 16;   // rhs chunk staged in shared memory

// dA[i, j] = alpha * sum_r P[i, r] * Q[j, r]   (P: n x k, Q: n x k, fp64)
__global__ void __launch_bounds__(256)
outer_kernel(int64_t n, int64_t k, double alpha, const double* __restrict__ P,
             int64_t ldp, const double* __restrict__ Q, int64_t ldq,
             float* __restrict__ dA, int64_t ldda) {
  __shared__ double ps[OR][OT];
  __shared__ double qs[OR][OT];
  const int tid = threadIdx.x, tx = tid % 16, ty = tid / 16;
  const int64_t i0 = (int64_t)blockIdx.x * OT, j0 = (int64_t)blockIdx.y * OT;
  double acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b] = 0.0;
  for (int64_t r0 = 0; r0 < k; r0 += OR) {
    for (int e = tid; e < OR * OT; e += 256) {
      const int ii = e % OT, rr = e / OT;
      const int64_t r = r0 + rr;
      ps[rr][ii] = (r < k && i0 + ii < n) ? P[i0 + ii + r * ldp] : 0.0;
      qs[rr][ii] = (r < k && j0 + ii < n) ? Q[j0 + ii + r * ldq] : 0.0;
    }
    __syncthreads();
#pragma unroll
    for (int rr = 0; rr < OR; ++rr) {
      double p[4], q[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) p[a] = ps[rr][tx * 4 + a];
#pragma unroll
      for (int b = 0; b < 4; ++b) q[b] = qs[rr][ty * 4 + b];
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] = fma(p[a], q[b], acc[a][b]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const int64_t i = i0 + tx * 4 + a, j = j0 + ty * 4 + b;
      if (i < n && j < n) dA[i + j * ldda] = (float)(alpha * acc[a][b]);
    }
}

// r = b - A^T x, one warp per column of A (coalesced), lane-strided partial
// sums reduced in a fixed tree; maxes as in the forward residual.
__global__ void __launch_bounds__(256)
residual_t_kernel(int64_t n, const float* __restrict__ A, int64_t lda,
                  const double* __restrict__ b, const double* __restrict__ x,
                  double* __restrict__ r, unsigned long long* __restrict__ maxes) {
  const int lane = threadIdx.x & 31;
  const int64_t i = ((int64_t)blockIdx.x * 256 + threadIdx.x) / 32;
  double ri = 0.0, xi = 0.0, bi = 0.0;
  if (i < n) {
    const float* col = A + i * lda;
    double p = 0.0;
    for (int64_t j = lane; j < n; j += 32) p = fma((double)col[j], x[j], p);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) p += __shfl_xor_sync(0xffffffffu, p, o);
    bi = b[i];
    ri = bi - p;
    xi = x[i];
    if (lane == 0) r[i] = ri;
  }
  if (lane == 0 && i < n) {
    atomicMax(&maxes[0], (unsigned long long)__double_as_longlong(fabs(ri)));
    atomicMax(&maxes[1], (unsigned long long)__double_as_longlong(fabs(xi)));
    atomicMax(&maxes[2], (unsigned long long)__double_as_longlong(fabs(bi)));
  }
}

// ||A^T||_inf = max column sum of |A|
__global__ void __launch_bounds__(256)
colsum_kernel(int64_t n, const float* __restrict__ A, int64_t lda,
              unsigned long long* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  const int64_t i = ((int64_t)blockIdx.x * 256 + threadIdx.x) / 32;
  if (i >= n) return;
  const float* col = A + i * lda;
  double p = 0.0;
  for (int64_t j = lane; j < n; j += 32) p += fabs((double)col[j]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) p += __shfl_xor_sync(0xffffffffu, p, o);
  if (lane == 0) atomicMax(out, (unsigned long long)__double_as_longlong(p));
}

}  // namespace

lu_status launch_outer(cudaStream_t st, int64_t n, int64_t k, double alpha,
                       const double* P, int64_t ldp, const double* Q, int64_t ldq,
                       float* dA, int64_t ldda) {
  if (n <= 0) return LU_SUCCESS;
  dim3 g((unsigned)ceil_div(n, OT), (unsigned)ceil_div(n, OT));
  outer_kernel<<<g, 256, 0, st>>>(n, k, alpha, P, ldp, Q, ldq, dA, ldda);
  LUB_LAUNCH_CHECK();
  return LU_SUCCESS;
}

lu_status launch_residual_t(cudaStream_t st, int64_t n, const float* A,
                            int64_t lda, const double* b, const double* x,
                            double* r, unsigned long long* maxes) {
  LUB_CUDA_TRY(cudaMemsetAsync(maxes, 0, 3 * sizeof(unsigned long long), st));
  residual_t_kernel<<<(unsigned)ceil_div(n * 32, 256), 256, 0, st>>>(n, A, lda, b, x, r, maxes);
  LUB_LAUNCH_CHECK();
  return LU_SUCCESS;
}

lu_status launch_norm_one(cudaStream_t st, int64_t n, const float* A,
                          int64_t lda, unsigned long long* out) {
  LUB_CUDA_TRY(cudaMemsetAsync(out, 0, sizeof(unsigned long long), st));
  colsum_kernel<<<(unsigned)ceil_div(n * 32, 256), 256, 0, st>>>(n, A, lda, out);
  LUB_LAUNCH_CHECK();
  return LU_SUCCESS;
}

}  // namespace lub

using namespace lub;

extern "C" {

LU_API lu_status lu_adjoint_workspace_size(int64_t n, int64_t nrhs, size_t* bytes) {
  if (n < 0 || nrhs < 0 || !bytes) return LU_ERR_INVALID_ARG;
  size_t rw = 0;
  LUB_TRY(lu_refine_ex_workspace_size(n, nrhs, &rw));
  *bytes = align_up((size_t)n * (size_t)nrhs * 8, 256) + rw;
  return LU_SUCCESS;
}

LU_API lu_status lu_adjoint_c(lu_stream_t stream, int64_t n, int64_t nrhs,
                              const float* d_a, int64_t lda, const float* d_lu,
                              int64_t ldlu, const double* d_x, int64_t ldx,
                              double* d_g, int64_t ldg, float* d_da, int64_t ldda,
                              double tol, int max_iter, int* iters, double* berr,
                              void* workspace, size_t ws_bytes) {
  if (n < 0 || nrhs < 0 || ldlu < std::max<int64_t>(1, n) ||
      ldx < std::max<int64_t>(1, n) || ldg < std::max<int64_t>(1, n) ||
      (d_da && ldda < std::max<int64_t>(1, n)) ||
      (d_a && (lda < std::max<int64_t>(1, n) || max_iter < 0 || !(tol >= 0.0))))
    return LU_ERR_INVALID_ARG;
  if (iters) *iters = 0;
  if (berr) *berr = 0.0;
  if (n == 0 || nrhs == 0) return LU_SUCCESS;
  if (!d_lu || !d_x || !d_g) return LU_ERR_INVALID_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  lu_status s = LU_SUCCESS;
  if (!d_a) {
    // dB = A^-T G = L^-T U^-T G, in place in d_g
    LUB_TRY(lu_solve_c(stream, n, d_lu, ldlu, d_g, ldg, nrhs, 1));
  } else {
    // refined: keep G as the right-hand side, refine A^T dB = G into d_g
    size_t need = 0;
    LUB_TRY(lu_adjoint_workspace_size(n, nrhs, &need));
    if (workspace && ws_bytes < need) return LU_ERR_WORKSPACE;
    void* ws = workspace;
    bool owned = false;
    if (!ws) {
      if (pool_malloc_async((void**)&ws, need, st) != cudaSuccess) return LU_ERR_ALLOC;
      owned = true;
    }
    double* g0 = static_cast<double*>(ws);
    const size_t off = align_up((size_t)n * (size_t)nrhs * 8, 256);
    if (cudaMemcpy2DAsync(g0, (size_t)n * 8, d_g, (size_t)ldg * 8, (size_t)n * 8,
                          (size_t)nrhs, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
      s = LU_ERR_CUDA;
    if (s == LU_SUCCESS)
      s = lu_refine_ex_c(stream, n, nrhs, d_a, lda, d_lu, ldlu, g0, n, d_g, ldg, 1,
                         tol, max_iter, iters, berr, static_cast<char*>(ws) + off,
                         need - off);
    if (owned) cudaFreeAsync(ws, st);
    if (s != LU_SUCCESS && s != LU_ERR_NOT_CONVERGED) return s;
  }
  // dA = -dB X^T
  if (d_da) LUB_TRY(launch_outer(st, n, nrhs, -1.0, d_g, ldg, d_x, ldx, d_da, ldda));
  return s;
}

}  // extern "C"
