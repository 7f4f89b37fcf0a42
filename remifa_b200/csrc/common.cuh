// Shared helpers for the sm_100a kernels and the C-ABI layer.
#pragma once

#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cuda_bf16.h>
#include <cuda_fp8.h>
#include <cstdint>
#include <cstdio>

#include "lu_b200.h"

namespace lub {

// Sentinel stored in the "first bad pivot" word before a factorization.
constexpr int kNoBadPivot = 0x7f7f7f7f;

#define LUB_CUDA_TRY(expr)                                              \
  do {                                                                  \
    cudaError_t _e = (expr);                                            \
    if (_e != cudaSuccess) {                                            \
      ::lub::record_cuda_error(_e, #expr, __FILE__, __LINE__);          \
      return LU_ERR_CUDA;                                               \
    }                                                                   \
  } while (0)

#define LUB_LAUNCH_CHECK()                                              \
  do {                                                                  \
    cudaError_t _e = cudaGetLastError();                                \
    if (_e != cudaSuccess) {                                            \
      ::lub::record_cuda_error(_e, "kernel launch", __FILE__, __LINE__); \
      return LU_ERR_CUDA;                                               \
    }                                                                   \
    ::lub::count_launch();                                              \
  } while (0)

#define LUB_TRY(expr)                       \
  do {                                      \
    lu_status _s = (expr);                  \
    if (_s != LU_SUCCESS) return _s;        \
  } while (0)

// Store a plain message for lu_last_error (this thread).
void record_message(const char* msg);
void record_cuda_error(cudaError_t e, const char* what, const char* file,
                       int line);
// Counts one kernel launch of this library (profile.cu).
void count_launch();

inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }
inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// Number of SMs of the current device (cached per device).
int sm_count();

// Stream-ordered allocation from the library's own memory pool on the
// current device (misc.cu).  Freed blocks (cudaFreeAsync) stay reserved in
// the pool for the next call instead of going back to the driver, so calls
// that leave the workspace to the library do not map and unmap up to
// gigabytes each time; lu_trim_memory_c hands them back.
cudaError_t pool_malloc_async(void** p, size_t bytes, cudaStream_t st);

// ---- device helpers -------------------------------------------------------

// Asynchronous 4-byte global -> shared copy (no register round trip, so a
// thread can have hundreds in flight).  Complete with cp_async_wait_all().
__device__ __forceinline__ void cp_async4(float* smem_dst, const float* gsrc) {
  const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(smem_dst));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(gsrc) : "memory");
}
// 16-byte variant: both addresses 16-byte aligned.
__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gsrc) {
  const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(smem_dst));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

// Correctly rounded 1/d (IEEE round to nearest even).  For normal d with
// 2^-125 < |d| < 2^125: the hardware approximation rcp.approx.ftz.f32 refined
// by Newton-Raphson steps in fused multiply-adds, e = 1 - d y (exact when y
// is within an ulp), y' = y + e y -- the FMA reciprocal iteration published
// by Markstein ("Computation of elementary functions on the IBM RISC
// System/6000 processor", IBM J. Res. Dev. 34(1), 1990).  Two steps leave an
// error far below the distance from 1/d to the nearest rounding boundary.
// Other inputs (zero, subnormal, huge, inf, nan) take __frcp_rn.  Checked
// against __frcp_rn for every float bit pattern (lu_selfcheck_rcp_c).
__device__ __forceinline__ float rcp_rn(float d) {
  const float a = fabsf(d);
  if (a > 0x1p-125f && a < 0x1p125f) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(d));
    float e = __fmaf_rn(-d, y, 1.0f);
    y = __fmaf_rn(e, y, y);
    e = __fmaf_rn(-d, y, 1.0f);
    return __fmaf_rn(e, y, y);
  }
  return __frcp_rn(d);
}

// rcp_rn without the range test, for callers that check the range of the
// pivots afterwards (2^-125 < |d| < 2^125) and redo the work otherwise.
__device__ __forceinline__ float rcp_rn_unchecked(float d) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(d));
  float e = __fmaf_rn(-d, y, 1.0f);
  y = __fmaf_rn(e, y, y);
  e = __fmaf_rn(-d, y, 1.0f);
  return __fmaf_rn(e, y, y);
}

// Factor a full 8x8 tile (column-major at T, leading dimension LD, 16-byte
// aligned columns) in registers with the reference's operation order:
// 1/d, the column below scaled, fused a - l*u for the rest
// (src/lu_nopiv.cu:123-171).  The pivot chain carries no branch: the
// pivots are range-checked afterwards, and if any lies outside
// (2^-125, 2^125) -- zero, subnormal, huge or non-finite -- nothing is
// written and false is returned, so the caller can redo the tile on the
// exact slow path (which also reports the bad pivot).
__device__ __forceinline__ bool factor_tile8_fast(float* T, int LD, float* inv) {
  float v[8][8];  // v[c][r]: tile column c
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    const float4 a = *reinterpret_cast<const float4*>(T + c * LD);
    const float4 b = *reinterpret_cast<const float4*>(T + c * LD + 4);
    v[c][0] = a.x; v[c][1] = a.y; v[c][2] = a.z; v[c][3] = a.w;
    v[c][4] = b.x; v[c][5] = b.y; v[c][6] = b.z; v[c][7] = b.w;
  }
  float dk[8], ivk[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    dk[k] = v[k][k];
    ivk[k] = rcp_rn_unchecked(dk[k]);
#pragma unroll
    for (int r = k + 1; r < 8; ++r) v[k][r] = __fmul_rn(v[k][r], ivk[k]);
#pragma unroll
    for (int c = k + 1; c < 8; ++c)
#pragma unroll
      for (int r = k + 1; r < 8; ++r) v[c][r] = __fmaf_rn(-v[k][r], v[c][k], v[c][r]);
  }
  bool safe = true;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const float a = fabsf(dk[k]);
    safe = safe && a > 0x1p-125f && a < 0x1p125f;
  }
  if (!safe) return false;
#pragma unroll
  for (int k = 0; k < 8; ++k) inv[k] = ivk[k];
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    *reinterpret_cast<float4*>(T + c * LD) = make_float4(v[c][0], v[c][1], v[c][2], v[c][3]);
    *reinterpret_cast<float4*>(T + c * LD + 4) = make_float4(v[c][4], v[c][5], v[c][6], v[c][7]);
  }
  return true;
}

// Record the 1-based global index of a zero / non-finite pivot.
__device__ __forceinline__ void note_pivot(float d, int64_t col0,
                                           int* first_bad) {
  if (first_bad != nullptr && !(fabsf(d) > 0.0f && isfinite(d)))
    atomicMin(first_bad, (int)(col0 + 1));
}

}  // namespace lub
