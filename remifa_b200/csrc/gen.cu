// Seeded, counter-based generator of diagonally dominant test matrices.
//
// Each entry is a pure function of (seed, i, j), so a matrix of any size is
// produced in parallel and is bit-identical to the CPU generator used by the
// tests.  The reference generates its inputs on the host with
// std::default_random_engine (tests/genmat.hxx:69-102,
// tests/common.hxx:298-319); the benchmark shapes (n up to 32768) are
// generated on the device instead.
//
// kind 0: r_ij = q * 2^-23, q uniform in [-2^23, 2^23)      (U[-1,1))
// kind 1: r_ij = q * 2^-21 / sqrt(n), q = sum of twelve 21-bit uniforms,
//         centred (Irwin-Hall, ~N(0,1)/sqrt(n))
// kind 2: r_ij = -|kind 1| (every off-diagonal entry negative: with the
//         dominant diagonal an M-matrix, A 1 = (alpha - 1) diag(A) 1 / alpha,
//         so kappa_2(A) ~ 1 / (alpha - 1): the dominance sets the condition)
// a_ij = r_ij for i != j;  a_ii = alpha * sum_{j != i} |r_ij| (exact integer
// row sum, then two fp64 multiplies rounded once to fp32); all entries
// times 2^kscale; row i times 2^-round(gamma_bits * i / (n - 1)).
#include "common.cuh"
#include "kernels.cuh"

namespace lub {
namespace {

// splitmix64 finaliser (Steele, Lea and Flood, 2014).
__device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__device__ __forceinline__ int32_t sample_q(uint64_t seedmix, uint64_t i,
                                            uint64_t j, int kind) {
  uint64_t h = mix64(((i << 32) | (j & 0xffffffffull)) ^ seedmix);
  if (kind == 0) return (int32_t)(h >> 40) - (1 << 23);
  int64_t s = 0;
#pragma unroll
  for (int w = 0; w < 4; ++w) {
    s += (int64_t)(h & 0x1fffff);
    s += (int64_t)((h >> 21) & 0x1fffff);
    s += (int64_t)((h >> 42) & 0x1fffff);
    h = mix64(h);
  }
  const int32_t q = (int32_t)(s - 6ll * (1ll << 21));
  return kind == 2 ? (q < 0 ? q : -q) : q;
}

__device__ __forceinline__ int row_shift(double gamma_bits, int64_t i, int64_t n) {
  if (gamma_bits == 0.0 || n <= 1) return 0;
  return -(int)__double2ll_rn(__ddiv_rn(__dmul_rn(gamma_bits, (double)i), (double)(n - 1)));
}

constexpr int kColsPerBlock = 512;

__global__ void gen_offdiag_kernel(int64_t n, float* __restrict__ a, int64_t lda,
                                   uint64_t seedmix, int kind, float scale,
                                   int kscale, double gamma_bits,
                                   unsigned long long* __restrict__ rowsum) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int shift = row_shift(gamma_bits, i, n);
  const int64_t j0 = (int64_t)blockIdx.y * kColsPerBlock;
  const int64_t j1 = (n < j0 + kColsPerBlock) ? n : j0 + kColsPerBlock;
  unsigned long long s = 0;
  for (int64_t j = j0; j < j1; ++j) {
    if (j == i) continue;
    const int32_t q = sample_q(seedmix, (uint64_t)i, (uint64_t)j, kind);
    s += (unsigned long long)(q < 0 ? -(int64_t)q : (int64_t)q);
    const float v = __fmul_rn((float)q, scale);
    a[i + j * lda] = ldexpf(ldexpf(v, kscale), shift);
  }
  atomicAdd(&rowsum[i], s);
}

__global__ void gen_diag_kernel(int64_t n, float* __restrict__ a, int64_t lda,
                                float scale, double alpha, int kscale,
                                double gamma_bits,
                                const unsigned long long* __restrict__ rowsum) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float d = __double2float_rn(
      __dmul_rn(__dmul_rn(alpha, (double)rowsum[i]), (double)scale));
  a[i + i * lda] = ldexpf(ldexpf(d, kscale), row_shift(gamma_bits, i, n));
}

// One CTA per matrix of a batch (n <= 1024): thread per row.
__global__ void __launch_bounds__(256)
gen_batch_kernel(float* const* __restrict__ ptrs, const int32_t* __restrict__ ns,
                 const int32_t* __restrict__ ldas, uint64_t seed, int kind,
                 double alpha) {
  const int mat = blockIdx.x;
  const int64_t n = ns[mat];
  const int64_t lda = ldas ? (int64_t)ldas[mat] : n;
  float* a = ptrs[mat];
  const uint64_t seedmix = mix64(seed + (uint64_t)mat);
  const float scale =
      kind == 0 ? 0x1p-23f : (float)(0x1p-21 / sqrt((double)n));
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
    unsigned long long s = 0;
    for (int64_t j = 0; j < n; ++j) {
      if (j == i) continue;
      const int32_t q = sample_q(seedmix, (uint64_t)i, (uint64_t)j, kind);
      s += (unsigned long long)(q < 0 ? -(int64_t)q : (int64_t)q);
      a[i + j * lda] = __fmul_rn((float)q, scale);
    }
    a[i + i * lda] = __double2float_rn(__dmul_rn(__dmul_rn(alpha, (double)s), (double)scale));
  }
}

uint64_t host_mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

}  // namespace

lu_status launch_gen_matrix(cudaStream_t st, int64_t n, float* a, int64_t lda,
                            uint64_t seed, int kind, double alpha, int kscale,
                            double gamma_bits) {
  if (n < 0 || lda < std::max<int64_t>(1, n) || (kind < 0 || kind > 2))
    return LU_ERR_INVALID_ARG;
  if (n == 0) return LU_SUCCESS;
  if (a == nullptr) return LU_ERR_INVALID_ARG;
  const float scale =
      kind == 0 ? ldexpf(1.0f, -23)
                : (float)(ldexp(1.0, -21) / std::sqrt((double)n));
  unsigned long long* rowsum = nullptr;
  LUB_CUDA_TRY(pool_malloc_async((void**)&rowsum, n * sizeof(unsigned long long), st));
  LUB_CUDA_TRY(cudaMemsetAsync(rowsum, 0, n * sizeof(unsigned long long), st));
  const uint64_t seedmix = host_mix64(seed);
  dim3 grid((unsigned)ceil_div(n, 256), (unsigned)ceil_div(n, kColsPerBlock));
  gen_offdiag_kernel<<<grid, 256, 0, st>>>(n, a, lda, seedmix, kind, scale,
                                           kscale, gamma_bits, rowsum);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) {
    count_launch();
    gen_diag_kernel<<<(unsigned)ceil_div(n, 256), 256, 0, st>>>(
        n, a, lda, scale, alpha, kscale, gamma_bits, rowsum);
    e = cudaGetLastError();
    if (e == cudaSuccess) count_launch();
  }
  cudaFreeAsync(rowsum, st);
  if (e != cudaSuccess) {
    record_cuda_error(e, "gen kernels", __FILE__, __LINE__);
    return LU_ERR_CUDA;
  }
  return LU_SUCCESS;
}

lu_status launch_gen_batch(cudaStream_t st, int64_t batch, float* const* ptrs,
                           const int32_t* ns, const int32_t* ldas, uint64_t seed,
                           int kind, double alpha) {
  if (batch < 0 || (kind < 0 || kind > 2) || batch > INT32_MAX) return LU_ERR_INVALID_ARG;
  if (batch == 0) return LU_SUCCESS;
  if (!ptrs || !ns) return LU_ERR_INVALID_ARG;
  gen_batch_kernel<<<(unsigned)batch, 256, 0, st>>>(ptrs, ns, ldas, seed, kind, alpha);
  LUB_LAUNCH_CHECK();
  return LU_SUCCESS;
}

}  // namespace lub

extern "C" LU_API lu_status lu_gen_batch_c(lu_stream_t stream, int64_t batch,
                                           float* const* d_ptrs, const int32_t* d_n,
                                           const int32_t* d_lda, uint64_t seed, int kind,
                                           double alpha) {
  return lub::launch_gen_batch((cudaStream_t)stream, batch, d_ptrs, d_n, d_lda, seed,
                               kind, alpha);
}
