// Batched solves and adjoint for the factors a batch plan produced (new; the
// reference has neither a batch nor a derivative).
//
// One warp per (matrix, right-hand side): the warp keeps b, x and the
// residual of its column in shared memory (fp64) and works down the
// triangles with the fp32 factors read straight from global memory:
//   L x = b, U x = y   : column (axpy) form, column j of the factor read
//                        coalesced by the 32 lanes;
//   U^T z = g, L^T y = z: dot form, column j again, lane partial sums reduced
//                        in a fixed shuffle tree (deterministic).
// With the original fp32 matrices given, refine_iters rounds of FP64
// refinement follow: r = b - op(A) x in fp64, x += op(LU)^-1 r.
// The adjoint of X = A^-1 B: dB = A^-T G (the transposed solve above, in
// place in G) and dA = -dB X^T (fp64 dot products, stored fp32).
#include "common.cuh"
#include "kernels.cuh"

#include <algorithm>

struct lu_batch_plan_t;

namespace lub {

// plan accessors (batch.cu)
int64_t batch_plan_size(const lu_batch_plan_t* p);
const int32_t* batch_plan_dev_n(const lu_batch_plan_t* p);
int batch_plan_nmax(const lu_batch_plan_t* p);

namespace {

constexpr int kWarpsPerCta = 4;

// x (shared, fp64, length n) <- L^-1 x, L unit lower (fp32, column-major).
__device__ __forceinline__ void lower_solve(const float* __restrict__ F, int64_t ld,
                                            int n, double* x) {
  const int lane = threadIdx.x & 31;
  for (int j = 0; j < n - 1; ++j) {
    __syncwarp();
    const double xj = x[j];
    const float* col = F + (int64_t)j * ld;
    for (int i = j + 1 + lane; i < n; i += 32) x[i] = fma(-(double)col[i], xj, x[i]);
  }
  __syncwarp();
}

// x <- U^-1 x, U upper with its diagonal (column form, bottom up).
__device__ __forceinline__ void upper_solve(const float* __restrict__ F, int64_t ld,
                                            int n, double* x) {
  const int lane = threadIdx.x & 31;
  for (int j = n - 1; j >= 0; --j) {
    __syncwarp();
    const float* col = F + (int64_t)j * ld;
    const double xj = x[j] / (double)col[j];
    __syncwarp();
    if (lane == 0) x[j] = xj;
    for (int i = lane; i < j; i += 32) x[i] = fma(-(double)col[i], xj, x[i]);
  }
  __syncwarp();
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// x <- U^-T x (dot form, top down: x_j = (x_j - U[0:j, j] . x[0:j]) / U_jj).
__device__ __forceinline__ void upper_t_solve(const float* __restrict__ F, int64_t ld,
                                              int n, double* x) {
  const int lane = threadIdx.x & 31;
  for (int j = 0; j < n; ++j) {
    const float* col = F + (int64_t)j * ld;
    double p = 0.0;
    for (int i = lane; i < j; i += 32) p = fma((double)col[i], x[i], p);
    p = warp_sum(p);
    if (lane == 0) x[j] = (x[j] - p) / (double)col[j];
    __syncwarp();
  }
}

// x <- L^-T x (dot form, bottom up: x_j = x_j - L[j+1:n, j] . x[j+1:n]).
__device__ __forceinline__ void lower_t_solve(const float* __restrict__ F, int64_t ld,
                                              int n, double* x) {
  const int lane = threadIdx.x & 31;
  for (int j = n - 2; j >= 0; --j) {
    const float* col = F + (int64_t)j * ld;
    double p = 0.0;
    for (int i = j + 1 + lane; i < n; i += 32) p = fma((double)col[i], x[i], p);
    p = warp_sum(p);
    if (lane == 0) x[j] = x[j] - p;
    __syncwarp();
  }
}

__device__ __forceinline__ void solve(const float* F, int64_t ld, int n, double* x,
                                      bool trans) {
  if (!trans) {
    lower_solve(F, ld, n, x);
    upper_solve(F, ld, n, x);
  } else {
    upper_t_solve(F, ld, n, x);
    lower_t_solve(F, ld, n, x);
  }
}

// r = b - op(A) x (A fp32, fp64 arithmetic).
__device__ __forceinline__ void residual(const float* __restrict__ A, int64_t ld, int n,
                                         const double* b, const double* x, double* r,
                                         bool trans) {
  const int lane = threadIdx.x & 31;
  if (!trans) {
    for (int i = lane; i < n; i += 32) r[i] = b[i];
    for (int j = 0; j < n; ++j) {
      __syncwarp();
      const double xj = x[j];
      const float* col = A + (int64_t)j * ld;
      for (int i = lane; i < n; i += 32) r[i] = fma(-(double)col[i], xj, r[i]);
    }
  } else {
    for (int j = 0; j < n; ++j) {
      const float* col = A + (int64_t)j * ld;
      double p = 0.0;
      for (int i = lane; i < n; i += 32) p = fma((double)col[i], x[i], p);
      p = warp_sum(p);
      if (lane == 0) r[j] = b[j] - p;
    }
  }
  __syncwarp();
}

struct SolveArgs {
  const float* const* lu;
  const int32_t* ldlu;
  const float* const* a;    // original matrices (refinement), or null
  const int32_t* lda;
  double* const* x;         // n_i x nrhs, ld n_i: b on entry, x on exit
  const int32_t* n;
  int64_t batch;
  int nrhs;
  int trans;
  int iters;
  int nmax;
};

__global__ void __launch_bounds__(32 * kWarpsPerCta)
batch_solve_kernel(SolveArgs s) {
  extern __shared__ double sh[];
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double* xb = sh + (size_t)wid * 3 * s.nmax;
  double* bb = xb + s.nmax;
  double* rb = bb + s.nmax;
  const int64_t items = s.batch * s.nrhs;
  for (int64_t it = (int64_t)blockIdx.x * kWarpsPerCta + wid; it < items;
       it += (int64_t)gridDim.x * kWarpsPerCta) {
    const int64_t m = it / s.nrhs;
    const int c = (int)(it - m * s.nrhs);
    const int n = s.n[m];
    const float* F = s.lu[m];
    const int64_t ldf = s.ldlu ? s.ldlu[m] : n;
    double* xg = s.x[m] + (int64_t)c * n;
    for (int i = lane; i < n; i += 32) {
      xb[i] = xg[i];
      bb[i] = xg[i];
    }
    __syncwarp();
    solve(F, ldf, n, xb, s.trans != 0);
    if (s.a) {
      const float* A = s.a[m];
      const int64_t lda = s.lda ? s.lda[m] : n;
      for (int k = 0; k < s.iters; ++k) {
        residual(A, lda, n, bb, xb, rb, s.trans != 0);
        solve(F, ldf, n, rb, s.trans != 0);
        for (int i = lane; i < n; i += 32) xb[i] += rb[i];
        __syncwarp();
      }
    }
    for (int i = lane; i < n; i += 32) xg[i] = xb[i];
    __syncwarp();
  }
}

// dA_m[i, j] = -sum_r dB_m[i, r] X_m[j, r], one CTA per matrix.
__global__ void __launch_bounds__(256)
batch_outer_kernel(const double* const* __restrict__ db, const double* const* __restrict__ x,
                   float* const* __restrict__ da, const int32_t* __restrict__ ldda,
                   const int32_t* __restrict__ ns, int nrhs) {
  const int m = blockIdx.x;
  const int n = ns[m];
  const int64_t ld = ldda ? (int64_t)ldda[m] : n;
  const double* G = db[m];
  const double* X = x[m];
  float* D = da[m];
  for (int64_t e = threadIdx.x; e < (int64_t)n * n; e += blockDim.x) {
    const int j = (int)(e / n), i = (int)(e - (int64_t)j * n);
    double acc = 0.0;
    for (int r = 0; r < nrhs; ++r)
      acc = fma(G[i + (int64_t)r * n], X[j + (int64_t)r * n], acc);
    D[i + j * ld] = (float)(-acc);
  }
}

lu_status launch_batch_solve(cudaStream_t st, const SolveArgs& s) {
  if (s.batch == 0 || s.nrhs == 0) return LU_SUCCESS;
  const size_t smem = (size_t)kWarpsPerCta * 3 * s.nmax * sizeof(double);
  LUB_CUDA_TRY(set_smem_limit((const void*)batch_solve_kernel, smem));
  const int64_t items = s.batch * s.nrhs;
  const int64_t grid = std::min<int64_t>((items + kWarpsPerCta - 1) / kWarpsPerCta,
                                         (int64_t)sm_count() * 16);
  batch_solve_kernel<<<(unsigned)grid, 32 * kWarpsPerCta, smem, st>>>(s);
  LUB_LAUNCH_CHECK();
  return LU_SUCCESS;
}

}  // namespace
}  // namespace lub

using namespace lub;

extern "C" {

LU_API lu_status lu_batch_solve_c(lu_batch_plan plan, lu_stream_t stream,
                                  const float* const* d_lu, const int32_t* d_ldlu,
                                  const float* const* d_a, const int32_t* d_lda,
                                  double* const* d_x, int32_t nrhs, int trans,
                                  int refine_iters) {
  if (!plan || nrhs < 0 || (trans != 0 && trans != 1) || refine_iters < 0)
    return LU_ERR_INVALID_ARG;
  const int64_t batch = batch_plan_size(plan);
  if (batch == 0 || nrhs == 0) return LU_SUCCESS;
  if (!d_lu || !d_x) return LU_ERR_INVALID_ARG;
  SolveArgs s;
  s.lu = d_lu;
  s.ldlu = d_ldlu;
  s.a = d_a;
  s.lda = d_lda;
  s.x = d_x;
  s.n = batch_plan_dev_n(plan);
  s.batch = batch;
  s.nrhs = nrhs;
  s.trans = trans;
  s.iters = d_a ? refine_iters : 0;
  s.nmax = batch_plan_nmax(plan);
  return launch_batch_solve((cudaStream_t)stream, s);
}

LU_API lu_status lu_batch_adjoint_c(lu_batch_plan plan, lu_stream_t stream,
                                    const float* const* d_lu, const int32_t* d_ldlu,
                                    const float* const* d_a, const int32_t* d_lda,
                                    double* const* d_x, double* const* d_g,
                                    float* const* d_da, const int32_t* d_ldda,
                                    int32_t nrhs, int refine_iters) {
  if (!plan || nrhs < 0 || refine_iters < 0) return LU_ERR_INVALID_ARG;
  const int64_t batch = batch_plan_size(plan);
  if (batch == 0 || nrhs == 0) return LU_SUCCESS;
  if (!d_lu || !d_x || !d_g) return LU_ERR_INVALID_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  LUB_TRY(lu_batch_solve_c(plan, stream, d_lu, d_ldlu, d_a, d_lda, d_g, nrhs, 1,
                           refine_iters));
  if (d_da) {
    batch_outer_kernel<<<(unsigned)batch, 256, 0, st>>>(d_g, d_x, d_da, d_ldda,
                                                        batch_plan_dev_n(plan), nrhs);
    LUB_LAUNCH_CHECK();
  }
  return LU_SUCCESS;
}

}  // extern "C"
