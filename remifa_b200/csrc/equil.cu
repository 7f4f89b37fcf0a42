// Equilibration by powers of two (new on the device; the reference
// equilibrates on the host with LAPACK geequb + laqge before factoring,
// tests/testing_lu_gpu.hxx:288-311).
//
// geequb's rule, restated: row scale r_i = 1 / 2^t(max_j |a_ij|), column
// scale c_j = 1 / 2^t(max_i r_i |a_ij|), with t(v) = trunc(log2 v) (toward
// zero) computed exactly from v's exponent, each clamped to
// [SMLNUM, 1 / SMLNUM]; rowcnd = max(rmin, SMLNUM) / min(rmax, BIGNUM) over
// the unclamped row maxima' powers (colcnd likewise); amax = max |a_ij|.
// laqge's rule: scale the rows when rowcnd < 0.1 or amax is outside
// [SMALL, LARGE] (SMALL = SMLNUM / ULP, LARGE = 1 / SMALL), the columns when
// colcnd < 0.1; the matrix becomes R A C in place.  Every scale is a power
// of two, so the scaled matrix is exact and its factors are exactly those
// of the original problem rescaled: A x = b <=> (R A C) (C^-1 x) = R b.
//
// Maxima are taken with integer atomicMax on the bit patterns of
// non-negative floats, so the result does not depend on scheduling.
#include "common.cuh"
#include "kernels.cuh"
#include "lu_b200.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <vector>

using namespace lub;

namespace {

constexpr int kEqCols = 256;  // columns per CTA of the row-maximum pass

// rmax_bits[i] = max over a column chunk of |a_ij| (atomicMax on bits)
__global__ void row_amax_kernel(int64_t n, const float* __restrict__ a, int64_t lda,
                                int* __restrict__ rmax_bits) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t j0 = (int64_t)blockIdx.y * kEqCols;
  const int64_t j1 = j0 + kEqCols < n ? j0 + kEqCols : n;
  float m = 0.0f;
  for (int64_t j = j0; j < j1; ++j) m = fmaxf(m, fabsf(a[i + j * lda]));
  atomicMax(&rmax_bits[i], __float_as_int(m));
}

// cmax_bits[j] = max_i |a_ij| * r_i (one CTA per column, fixed reduction)
__global__ void col_amax_kernel(int64_t n, const float* __restrict__ a, int64_t lda,
                                const float* __restrict__ r, int* __restrict__ cmax_bits) {
  __shared__ float red[256];
  const int64_t j = blockIdx.x;
  float m = 0.0f;
  for (int64_t i = threadIdx.x; i < n; i += 256)
    m = fmaxf(m, fabsf(a[i + j * lda]) * (r ? r[i] : 1.0f));  // r: a power of two
  red[threadIdx.x] = m;
  __syncthreads();
  for (int h = 128; h > 0; h >>= 1) {
    if (threadIdx.x < h) red[threadIdx.x] = fmaxf(red[threadIdx.x], red[threadIdx.x + h]);
    __syncthreads();
  }
  if (threadIdx.x == 0) cmax_bits[j] = __float_as_int(red[0]);
}

// a_ij *= r_i c_j (either may be null)
__global__ void scale_kernel(int64_t n, float* __restrict__ a, int64_t lda,
                             const float* __restrict__ r, const float* __restrict__ c) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float ri = r ? r[i] : 1.0f;
  for (int64_t j = blockIdx.y; j < n; j += gridDim.y) a[i + j * lda] *= ri * (c ? c[j] : 1.0f);
}

// The power of two geequb keeps for a maximum v > 0: 2^trunc(log2 v), the
// truncation toward zero taken from the exponent (v = m 2^e, m in [0.5, 1):
// log2 v lies in [e - 1, e), so trunc is e - 1 for v >= 1 or m = 0.5, else e).
int trunc_log2(float v) {
  int e = 0;
  const float m = std::frexp(v, &e);
  return (v >= 1.0f || m == 0.5f) ? e - 1 : e;
}

}  // namespace

extern "C" {

LU_API lu_status lu_equilibrate_c(lu_stream_t stream, int64_t n, float* d_a, int64_t lda,
                                  float* d_r, float* d_c, int force, char* equed,
                                  double* rowcnd, double* colcnd, double* amax) {
  if (n < 0 || lda < std::max<int64_t>(1, n) || !equed) return LU_ERR_INVALID_ARG;
  if (n > 0 && (!d_a || !d_r || !d_c)) return LU_ERR_INVALID_ARG;
  if (n > 0x7fffffffll) return LU_ERR_INVALID_ARG;
  *equed = 'N';
  if (rowcnd) *rowcnd = 1.0;
  if (colcnd) *colcnd = 1.0;
  if (amax) *amax = 0.0;
  if (n == 0) return LU_SUCCESS;
  int dev = 0, major = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev) != cudaSuccess ||
      major != 10)
    return LU_ERR_NO_DEVICE;
  cudaStream_t st = (cudaStream_t)stream;
  const float smlnum = FLT_MIN;  // slamch('S')
  const float bignum = 1.0f / smlnum;
  const float ulp = FLT_EPSILON;  // slamch('P') = eps * radix... per geequb's use
  // row maxima (into d_c, reused as scratch), read back
  int* rbits = reinterpret_cast<int*>(d_c);
  LUB_CUDA_TRY(cudaMemsetAsync(rbits, 0, (size_t)n * 4, st));
  dim3 g1((unsigned)ceil_div(n, 256), (unsigned)std::min<int64_t>(ceil_div(n, kEqCols), 65535));
  row_amax_kernel<<<g1, 256, 0, st>>>(n, d_a, lda, rbits);
  LUB_LAUNCH_CHECK();
  std::vector<float> h((size_t)n);
  LUB_CUDA_TRY(cudaMemcpyAsync(h.data(), rbits, (size_t)n * 4, cudaMemcpyDeviceToHost, st));
  LUB_CUDA_TRY(cudaStreamSynchronize(st));
  float am = 0.0f, rmin = bignum, rmax = 0.0f;
  std::vector<float> r((size_t)n);
  for (int64_t i = 0; i < n; ++i) {
    am = std::max(am, h[i]);
    const float p = h[i] > 0.0f ? std::ldexp(1.0f, trunc_log2(h[i])) : 0.0f;
    rmin = std::min(rmin, p);
    rmax = std::max(rmax, p);
    r[i] = p;
  }
  if (amax) *amax = am;
  if (rmin == 0.0f) return LU_SUCCESS;  // a zero row: geequb reports it, no scaling
  for (int64_t i = 0; i < n; ++i) r[i] = 1.0f / std::min(std::max(r[i], smlnum), bignum);
  const double rcnd = (double)std::max(rmin, smlnum) / (double)std::min(rmax, bignum);
  if (rowcnd) *rowcnd = rcnd;
  LUB_CUDA_TRY(cudaMemcpyAsync(d_r, r.data(), (size_t)n * 4, cudaMemcpyHostToDevice, st));
  // column maxima of R A
  int* cbits = reinterpret_cast<int*>(d_c);
  col_amax_kernel<<<(unsigned)n, 256, 0, st>>>(n, d_a, lda, d_r, cbits);
  LUB_LAUNCH_CHECK();
  LUB_CUDA_TRY(cudaMemcpyAsync(h.data(), cbits, (size_t)n * 4, cudaMemcpyDeviceToHost, st));
  LUB_CUDA_TRY(cudaStreamSynchronize(st));
  float cmin = bignum, cmax = 0.0f;
  std::vector<float> c((size_t)n);
  for (int64_t j = 0; j < n; ++j) {
    const float p = h[j] > 0.0f ? std::ldexp(1.0f, trunc_log2(h[j])) : 0.0f;
    cmin = std::min(cmin, p);
    cmax = std::max(cmax, p);
    c[j] = p;
  }
  if (cmin == 0.0f) return LU_SUCCESS;  // a zero column
  for (int64_t j = 0; j < n; ++j) c[j] = 1.0f / std::min(std::max(c[j], smlnum), bignum);
  const double ccnd = (double)std::max(cmin, smlnum) / (double)std::min(cmax, bignum);
  if (colcnd) *colcnd = ccnd;
  LUB_CUDA_TRY(cudaMemcpyAsync(d_c, c.data(), (size_t)n * 4, cudaMemcpyHostToDevice, st));
  // laqge's decision (THRESH = 0.1, SMALL = SMLNUM / ULP, LARGE = 1 / SMALL)
  const double small = (double)smlnum / (double)ulp, large = 1.0 / small;
  const bool rows = force || rcnd < 0.1 || am < small || am > large;
  const bool cols = force || ccnd < 0.1;
  if (rows || cols) {
    dim3 g2((unsigned)ceil_div(n, 256), (unsigned)std::min<int64_t>(n, 65535));
    scale_kernel<<<g2, 256, 0, st>>>(n, d_a, lda, rows ? d_r : nullptr, cols ? d_c : nullptr);
    LUB_LAUNCH_CHECK();
  }
  *equed = rows ? (cols ? 'B' : 'R') : (cols ? 'C' : 'N');
  // the scales not applied are reported as ones
  if (!rows) {
    std::fill(r.begin(), r.end(), 1.0f);
    LUB_CUDA_TRY(cudaMemcpyAsync(d_r, r.data(), (size_t)n * 4, cudaMemcpyHostToDevice, st));
  }
  if (!cols) {
    std::fill(c.begin(), c.end(), 1.0f);
    LUB_CUDA_TRY(cudaMemcpyAsync(d_c, c.data(), (size_t)n * 4, cudaMemcpyHostToDevice, st));
  }
  LUB_CUDA_TRY(cudaStreamSynchronize(st));
  return LU_SUCCESS;
}

}  // extern "C"
