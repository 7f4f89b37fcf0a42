// Precision conversion (cast copy) of a column-major m x n matrix.
//
// Replaces remifa::convert<TA,TAO> (src/convert.cu:324-387), whose kernel
// walks one row per thread across 64 columns with scalar 4-8 byte accesses.
// Here a thread converts 8 consecutive rows of one column with 16/32-byte
// vector loads and stores when the pointers and leading dimensions allow
// it, so the copy runs at HBM bandwidth.  Rounding is to nearest even
// (the reference's implicit float->half conversion, src/convert.cu:99-101);
// e4m3 saturates to +-448; an optional exact power-of-two scale is applied
// before rounding.
#include "common.cuh"
#include "kernels.cuh"

namespace lub {
namespace {

__device__ __forceinline__ float scale_f(float x, int s) {
  return s == 0 ? x : ldexpf(x, s);
}

template <typename TI, typename TO>
__device__ __forceinline__ TO convert_one(TI x, int s);

template <> __device__ __forceinline__ __half convert_one<float, __half>(float x, int s) {
  return __float2half_rn(scale_f(x, s));
}
template <> __device__ __forceinline__ __nv_bfloat16 convert_one<float, __nv_bfloat16>(float x, int s) {
  return __float2bfloat16_rn(scale_f(x, s));
}
template <> __device__ __forceinline__ __nv_fp8_e4m3 convert_one<float, __nv_fp8_e4m3>(float x, int s) {
  __nv_fp8_e4m3 r;
  r.__x = __nv_cvt_float_to_fp8(scale_f(x, s), __NV_SATFINITE, __NV_E4M3);
  return r;
}
template <> __device__ __forceinline__ float convert_one<float, float>(float x, int s) {
  return scale_f(x, s);
}
template <> __device__ __forceinline__ double convert_one<float, double>(float x, int s) {
  return ldexp((double)x, s);
}
template <> __device__ __forceinline__ float convert_one<__half, float>(__half x, int s) {
  return scale_f(__half2float(x), s);
}
template <> __device__ __forceinline__ double convert_one<__half, double>(__half x, int s) {
  return ldexp((double)__half2float(x), s);
}
template <> __device__ __forceinline__ __half convert_one<double, __half>(double x, int s) {
  return __double2half(ldexp(x, s));
}
template <> __device__ __forceinline__ float convert_one<double, float>(double x, int s) {
  return __double2float_rn(ldexp(x, s));
}

constexpr int kVec = 8;
constexpr int kThreads = 256;
constexpr int kRowsPerBlock = kThreads * kVec;

template <typename TI, typename TO, bool VEC>
__global__ void __launch_bounds__(kThreads)
convert_kernel(int64_t m, int64_t n, const TI* __restrict__ a, int64_t lda,
               TO* __restrict__ out, int64_t ldo, int s) {
  const int64_t i0 = ((int64_t)blockIdx.x * kThreads + threadIdx.x) * kVec;
  if (i0 >= m) return;
  for (int64_t j = blockIdx.y; j < n; j += gridDim.y) {
    const TI* src = a + i0 + j * lda;
    TO* dst = out + i0 + j * ldo;
    if (VEC && i0 + kVec <= m) {
      TI v[kVec];
      TO r[kVec];
      // 8 elements: one or two 16-byte loads depending on sizeof(TI)
      if constexpr (sizeof(TI) == 4) {
        const float4 x0 = reinterpret_cast<const float4*>(src)[0];
        const float4 x1 = reinterpret_cast<const float4*>(src)[1];
        memcpy(&v[0], &x0, 16);
        memcpy(&v[4], &x1, 16);
      } else if constexpr (sizeof(TI) == 2) {
        const float4 x0 = reinterpret_cast<const float4*>(src)[0];
        memcpy(&v[0], &x0, 16);
      } else {
#pragma unroll
        for (int q = 0; q < kVec; ++q) v[q] = src[q];
      }
#pragma unroll
      for (int q = 0; q < kVec; ++q) r[q] = convert_one<TI, TO>(v[q], s);
      if constexpr (sizeof(TO) == 4) {
        float4 y0, y1;
        memcpy(&y0, &r[0], 16);
        memcpy(&y1, &r[4], 16);
        reinterpret_cast<float4*>(dst)[0] = y0;
        reinterpret_cast<float4*>(dst)[1] = y1;
      } else if constexpr (sizeof(TO) == 2) {
        float4 y0;
        memcpy(&y0, &r[0], 16);
        reinterpret_cast<float4*>(dst)[0] = y0;
      } else if constexpr (sizeof(TO) == 1) {
        uint2 y0;
        memcpy(&y0, &r[0], 8);
        reinterpret_cast<uint2*>(dst)[0] = y0;
      } else {
#pragma unroll
        for (int q = 0; q < kVec; ++q) dst[q] = r[q];
      }
    } else {
      for (int q = 0; q < kVec && i0 + q < m; ++q) dst[q] = convert_one<TI, TO>(src[q], s);
    }
  }
}

template <typename TI, typename TO>
lu_status launch_typed(cudaStream_t st, int64_t m, int64_t n, const void* a,
                       int64_t lda, void* out, int64_t ldo, int s) {
  const bool vec =
      (lda % kVec == 0) && (ldo % kVec == 0) &&
      ((uintptr_t)a % (kVec * sizeof(TI) < 16 ? kVec * sizeof(TI) : 16) == 0) &&
      ((uintptr_t)out % (kVec * sizeof(TO) < 16 ? kVec * sizeof(TO) : 16) == 0);
  dim3 grid((unsigned)ceil_div(m, kRowsPerBlock),
            (unsigned)std::min<int64_t>(n, 65535));
  if (vec)
    convert_kernel<TI, TO, true><<<grid, kThreads, 0, st>>>(
        m, n, (const TI*)a, lda, (TO*)out, ldo, s);
  else
    convert_kernel<TI, TO, false><<<grid, kThreads, 0, st>>>(
        m, n, (const TI*)a, lda, (TO*)out, ldo, s);
  LUB_LAUNCH_CHECK();
  return LU_SUCCESS;
}

}  // namespace

lu_status launch_convert(cudaStream_t st, int64_t m, int64_t n, const void* a,
                         lu_dtype ta, int64_t lda, void* out, lu_dtype tout,
                         int64_t ldout, int s) {
  if (m < 0 || n < 0 || lda < std::max<int64_t>(1, m) ||
      ldout < std::max<int64_t>(1, m))
    return LU_ERR_INVALID_ARG;
  if (m == 0 || n == 0) return LU_SUCCESS;
  if (a == nullptr || out == nullptr) return LU_ERR_INVALID_ARG;
  if (ta == LU_F32) {
    switch (tout) {
      case LU_F16: return launch_typed<float, __half>(st, m, n, a, lda, out, ldout, s);
      case LU_BF16: return launch_typed<float, __nv_bfloat16>(st, m, n, a, lda, out, ldout, s);
      case LU_E4M3: return launch_typed<float, __nv_fp8_e4m3>(st, m, n, a, lda, out, ldout, s);
      case LU_F32: return launch_typed<float, float>(st, m, n, a, lda, out, ldout, s);
      case LU_F64: return launch_typed<float, double>(st, m, n, a, lda, out, ldout, s);
      default: return LU_ERR_UNSUPPORTED;
    }
  }
  if (ta == LU_F16) {
    if (tout == LU_F32) return launch_typed<__half, float>(st, m, n, a, lda, out, ldout, s);
    if (tout == LU_F64) return launch_typed<__half, double>(st, m, n, a, lda, out, ldout, s);
    return LU_ERR_UNSUPPORTED;
  }
  if (ta == LU_F64) {
    if (tout == LU_F16) return launch_typed<double, __half>(st, m, n, a, lda, out, ldout, s);
    if (tout == LU_F32) return launch_typed<double, float>(st, m, n, a, lda, out, ldout, s);
    return LU_ERR_UNSUPPORTED;
  }
  return LU_ERR_UNSUPPORTED;
}

}  // namespace lub
