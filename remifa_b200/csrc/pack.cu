// Operand packing for the tensor-core Schur update.
//
// The reference converts the fp32 L and U panels into an fp16 copy with the
// same column-major layout as A (src/lu_nopiv.hxx:155-164, convert kernel
// src/convert.cu:324-360).  The tensor core wants both operands K-major, so
// here the L21 panel is transposed while it is converted (row-major copy)
// and the U12 panel keeps its column-major layout with a compact leading
// dimension.  e4m3 copies carry one power-of-two scale per 128-row /
// 128-column tile, the largest that keeps the tile's max |x| <= 448; split
// fp16 copies (hi + lo) the same with bound 32768, which keeps the lo parts
// of all but the tile's tiniest entries normal fp16 numbers.
#include "common.cuh"
#include "kernels.cuh"
#include "tc_gemm.cuh"

namespace lub {
namespace {

template <typename T> __device__ __forceinline__ T to_low(float x);
template <> __device__ __forceinline__ __half to_low<__half>(float x) { return __float2half_rn(x); }
template <> __device__ __forceinline__ __nv_bfloat16 to_low<__nv_bfloat16>(float x) { return __float2bfloat16_rn(x); }
template <> __device__ __forceinline__ uint8_t to_low<uint8_t>(float x) {
  return (uint8_t)__nv_cvt_float_to_fp8(x, __NV_SATFINITE, __NV_E4M3);
}

__device__ __forceinline__ float to_f32(float x) { return x; }
__device__ __forceinline__ float to_f32(__half x) { return __half2float(x); }

constexpr int TA = 64;  // tile edge of the transposing pack

// S: source element type (fp32, or fp16 for the fp16-operand gemm entry,
// whose values pass through unchanged).
template <typename T, typename S = float>
__global__ void __launch_bounds__(256)
pack_a_kernel(int64_t M, int64_t K, const S* __restrict__ src, int64_t lds,
              T* __restrict__ dst, int64_t ldd, const int* __restrict__ scale) {
  __shared__ float tile[TA][TA + 1];  // [k][i]
  const int64_t i0 = (int64_t)blockIdx.x * TA;
  const int64_t k0 = (int64_t)blockIdx.y * TA;
  const int tid = threadIdx.x;
  // load: consecutive threads read consecutive rows of one column
  for (int q = tid; q < TA * TA; q += 256) {
    const int i = q % TA, k = q / TA;
    const int64_t gi = i0 + i, gk = k0 + k;
    tile[k][i] = (gi < M && gk < K) ? to_f32(src[gi + gk * lds]) : 0.0f;
  }
  __syncthreads();
  // store: consecutive threads write consecutive k of one row
  for (int q = tid; q < TA * TA; q += 256) {
    const int k = q % TA, i = q / TA;
    const int64_t gi = i0 + i, gk = k0 + k;
    if (gi < M && gk < K) {
      float x = tile[k][i];
      if (scale) x = ldexpf(x, scale[gi / 128]);
      dst[gi * ldd + gk] = to_low<T>(x);
    }
  }
}

// Split fp16: x = hi + lo with hi = rn(x), lo = rn(x - hi) (x - hi exact).
__device__ __forceinline__ void split16(float x, __half& hi, __half& lo) {
  hi = __float2half_rn(x);
  lo = __float2half_rn(__fsub_rn(x, __half2float(hi)));
}

// A: row i = [hi | hi | lo], segment stride kp, zeros in [K, kp).
__global__ void __launch_bounds__(256)
pack_a_split_kernel(int64_t M, int64_t K, int64_t kp, const float* __restrict__ src,
                    int64_t lds, __half* __restrict__ dst, int64_t ldd,
                    const int* __restrict__ scale) {
  __shared__ float tile[TA][TA + 1];  // [k][i]
  const int64_t i0 = (int64_t)blockIdx.x * TA;
  const int64_t k0 = (int64_t)blockIdx.y * TA;
  const int tid = threadIdx.x;
  for (int q = tid; q < TA * TA; q += 256) {
    const int i = q % TA, k = q / TA;
    const int64_t gi = i0 + i, gk = k0 + k;
    tile[k][i] = (gi < M && gk < K) ? src[gi + gk * lds] : 0.0f;
  }
  __syncthreads();
  for (int q = tid; q < TA * TA; q += 256) {
    const int k = q % TA, i = q / TA;
    const int64_t gi = i0 + i, gk = k0 + k;
    if (gi < M && gk < kp) {
      __half hi, lo;
      split16(ldexpf(tile[k][i], scale[gi / 128]), hi, lo);
      __half* row = dst + gi * ldd;
      row[gk] = hi;
      row[kp + gk] = hi;
      row[2 * kp + gk] = lo;
    }
  }
}

// B: column j = [hi ; lo ; hi], segment stride kp, zeros in [K, kp).
__global__ void __launch_bounds__(256)
pack_b_split_kernel(int64_t K, int64_t kp, int64_t N, const float* __restrict__ src,
                    int64_t lds, __half* __restrict__ dst, int64_t ldd,
                    const int* __restrict__ scale) {
  const int64_t k = (int64_t)blockIdx.x * 256 + threadIdx.x;
  if (k >= kp) return;
  for (int64_t j = blockIdx.y; j < N; j += gridDim.y) {
    const float x = k < K ? ldexpf(src[k + j * lds], scale[j / 128]) : 0.0f;
    __half hi, lo;
    split16(x, hi, lo);
    __half* col = dst + j * ldd;
    col[k] = hi;
    col[kp + k] = lo;
    col[2 * kp + k] = hi;
  }
}

template <typename T, typename S = float>
__global__ void __launch_bounds__(256)
pack_b_kernel(int64_t K, int64_t N, const S* __restrict__ src, int64_t lds,
              T* __restrict__ dst, int64_t ldd, const int* __restrict__ scale) {
  const int64_t k = (int64_t)blockIdx.x * 256 + threadIdx.x;
  if (k >= K) return;
  for (int64_t j = blockIdx.y; j < N; j += gridDim.y) {
    float x = to_f32(src[k + j * lds]);
    if (scale) x = ldexpf(x, scale[j / 128]);
    dst[k + j * ldd] = to_low<T>(x);
  }
}

// amax per tile, accumulated as the int bit pattern of a non-negative float
__global__ void __launch_bounds__(256)
amax_rows_kernel(int64_t M, int64_t K, const float* __restrict__ src,
                 int64_t lds, int* __restrict__ amax_bits) {
  // block: 128 rows x 32 columns; tile = blockIdx.x
  __shared__ float red[256];
  const int64_t i = (int64_t)blockIdx.x * 128 + (threadIdx.x % 128);
  const int64_t kb = (int64_t)blockIdx.y * 32;
  float m = 0.0f;
  if (i < M)
    for (int64_t k = kb + threadIdx.x / 128; k < K && k < kb + 32; k += 2)
      m = fmaxf(m, fabsf(src[i + k * lds]));
  red[threadIdx.x] = m;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] = fmaxf(red[threadIdx.x], red[threadIdx.x + w]);
    __syncthreads();
  }
  if (threadIdx.x == 0) atomicMax(&amax_bits[blockIdx.x], __float_as_int(red[0]));
}

__global__ void __launch_bounds__(256)
amax_cols_kernel(int64_t K, int64_t N, const float* __restrict__ src,
                 int64_t lds, int* __restrict__ amax_bits) {
  // block: one tile of 128 columns, rows strided by the block
  __shared__ float red[256];
  const int64_t j0 = (int64_t)blockIdx.x * 128;
  float m = 0.0f;
  for (int64_t j = j0 + blockIdx.y; j < N && j < j0 + 128; j += gridDim.y)
    for (int64_t k = threadIdx.x; k < K; k += 256) m = fmaxf(m, fabsf(src[k + j * lds]));
  red[threadIdx.x] = m;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] = fmaxf(red[threadIdx.x], red[threadIdx.x + w]);
    __syncthreads();
  }
  if (threadIdx.x == 0) atomicMax(&amax_bits[blockIdx.x], __float_as_int(red[0]));
}

// s = largest integer with amax * 2^s <= bound (0 for an all-zero or
// non-finite tile).
__global__ void amax_to_scale_kernel(int n, const int* __restrict__ amax_bits,
                                     int* __restrict__ scale, float bound) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const float a = __int_as_float(amax_bits[t]);
  int s = 0;
  if (a > 0.0f && isfinite(a)) {
    int e, eb;
    frexpf(a, &e);      // a in [2^(e-1), 2^e)
    frexpf(bound, &eb); // bound in [2^(eb-1), 2^eb)
    s = eb - 1 - e;     // a * 2^s < 2^(eb-1) <= bound
    while (ldexpf(a, s + 1) <= bound) ++s;
    while (ldexpf(a, s) > bound) --s;
  }
  scale[t] = s;
}

template <typename T>
lu_status pack_a_typed(cudaStream_t st, int64_t M, int64_t K, const float* src,
                       int64_t lds, void* dst, int64_t ldd, const int* scale) {
  dim3 grid((unsigned)ceil_div(M, TA), (unsigned)ceil_div(K, TA));
  pack_a_kernel<T><<<grid, 256, 0, st>>>(M, K, src, lds, (T*)dst, ldd, scale);
  LUB_LAUNCH_CHECK();
  return LU_SUCCESS;
}

template <typename T>
lu_status pack_b_typed(cudaStream_t st, int64_t K, int64_t N, const float* src,
                       int64_t lds, void* dst, int64_t ldd, const int* scale) {
  dim3 grid((unsigned)ceil_div(K, 256), (unsigned)std::min<int64_t>(N, 65535));
  pack_b_kernel<T><<<grid, 256, 0, st>>>(K, N, src, lds, (T*)dst, ldd, scale);
  LUB_LAUNCH_CHECK();
  return LU_SUCCESS;
}

}  // namespace

lu_status launch_pack_a(cudaStream_t st, TcOperand kind, int64_t M, int64_t K,
                        const float* src, int64_t lds, void* dst, int64_t ldd,
                        const int* scale) {
  if (M <= 0 || K <= 0) return LU_SUCCESS;
  switch (kind) {
    case TcOperand::F16: return pack_a_typed<__half>(st, M, K, src, lds, dst, ldd, nullptr);
    case TcOperand::BF16: return pack_a_typed<__nv_bfloat16>(st, M, K, src, lds, dst, ldd, nullptr);
    case TcOperand::E4M3: return pack_a_typed<uint8_t>(st, M, K, src, lds, dst, ldd, scale);
    case TcOperand::SPLIT16: {
      const int64_t kp = (K + 15) / 16 * 16;
      if (!scale || ldd < 3 * kp) return LU_ERR_INVALID_ARG;
      dim3 grid((unsigned)ceil_div(M, TA), (unsigned)ceil_div(kp, TA));
      pack_a_split_kernel<<<grid, 256, 0, st>>>(M, K, kp, src, lds, (__half*)dst, ldd, scale);
      LUB_LAUNCH_CHECK();
      return LU_SUCCESS;
    }
  }
  return LU_ERR_INVALID_ARG;
}

lu_status launch_pack_b(cudaStream_t st, TcOperand kind, int64_t K, int64_t N,
                        const float* src, int64_t lds, void* dst, int64_t ldd,
                        const int* scale) {
  if (N <= 0 || K <= 0) return LU_SUCCESS;
  switch (kind) {
    case TcOperand::F16: return pack_b_typed<__half>(st, K, N, src, lds, dst, ldd, nullptr);
    case TcOperand::BF16: return pack_b_typed<__nv_bfloat16>(st, K, N, src, lds, dst, ldd, nullptr);
    case TcOperand::E4M3: return pack_b_typed<uint8_t>(st, K, N, src, lds, dst, ldd, scale);
    case TcOperand::SPLIT16: {
      const int64_t kp = (K + 15) / 16 * 16;
      if (!scale || ldd < 3 * kp) return LU_ERR_INVALID_ARG;
      dim3 grid((unsigned)ceil_div(kp, 256), (unsigned)std::min<int64_t>(N, 65535));
      pack_b_split_kernel<<<grid, 256, 0, st>>>(K, kp, N, src, lds, (__half*)dst, ldd, scale);
      LUB_LAUNCH_CHECK();
      return LU_SUCCESS;
    }
  }
  return LU_ERR_INVALID_ARG;
}

lu_status launch_pack_a_f16(cudaStream_t st, int64_t M, int64_t K, const __half* src,
                            int64_t lds, __half* dst, int64_t ldd) {
  if (M <= 0 || K <= 0) return LU_SUCCESS;
  dim3 grid((unsigned)ceil_div(M, TA), (unsigned)ceil_div(K, TA));
  pack_a_kernel<__half, __half><<<grid, 256, 0, st>>>(M, K, src, lds, dst, ldd, nullptr);
  LUB_LAUNCH_CHECK();
  return LU_SUCCESS;
}

lu_status launch_pack_b_f16(cudaStream_t st, int64_t K, int64_t N, const __half* src,
                            int64_t lds, __half* dst, int64_t ldd) {
  if (N <= 0 || K <= 0) return LU_SUCCESS;
  dim3 grid((unsigned)ceil_div(K, 256), (unsigned)std::min<int64_t>(N, 65535));
  pack_b_kernel<__half, __half><<<grid, 256, 0, st>>>(K, N, src, lds, dst, ldd, nullptr);
  LUB_LAUNCH_CHECK();
  return LU_SUCCESS;
}

lu_status launch_scale_rowtiles(cudaStream_t st, int64_t M, int64_t K,
                                const float* src, int64_t lds, int* scale,
                                int* tmp, float bound) {
  if (M <= 0) return LU_SUCCESS;
  const int64_t tiles = ceil_div(M, 128);
  LUB_CUDA_TRY(cudaMemsetAsync(tmp, 0, tiles * sizeof(int), st));
  if (K > 0) {
    dim3 grid((unsigned)tiles, (unsigned)ceil_div(K, 32));
    amax_rows_kernel<<<grid, 256, 0, st>>>(M, K, src, lds, tmp);
    LUB_LAUNCH_CHECK();
  }
  amax_to_scale_kernel<<<(unsigned)ceil_div(tiles, 256), 256, 0, st>>>((int)tiles, tmp, scale,
                                                                      bound);
  LUB_LAUNCH_CHECK();
  return LU_SUCCESS;
}

lu_status launch_scale_coltiles(cudaStream_t st, int64_t K, int64_t N,
                                const float* src, int64_t lds, int* scale,
                                int* tmp, float bound) {
  if (N <= 0) return LU_SUCCESS;
  const int64_t tiles = ceil_div(N, 128);
  LUB_CUDA_TRY(cudaMemsetAsync(tmp, 0, tiles * sizeof(int), st));
  if (K > 0) {
    dim3 grid((unsigned)tiles, 16);
    amax_cols_kernel<<<grid, 256, 0, st>>>(K, N, src, lds, tmp);
    LUB_LAUNCH_CHECK();
  }
  amax_to_scale_kernel<<<(unsigned)ceil_div(tiles, 256), 256, 0, st>>>((int)tiles, tmp, scale,
                                                                      bound);
  LUB_LAUNCH_CHECK();
  return LU_SUCCESS;
}

}  // namespace lub
