// Panel kernels of the no-pivot LU (FP32 working precision).
//
// The reference factors each outer block column with an ib = 8 right-looking
// loop: per 8-column tile it factors the 8x8 diagonal tile (1/d then a
// multiply, fused rank-1 updates), eliminates the L rows below it and the U
// columns right of it, then applies a rank-8 GEMM update
// (src/lu_nopiv_inner_rl.hxx:104-196, src/lu_nopiv.cu:105-326).  Without
// pivoting the rows of L21 and the columns of U12 are independent of each
// other once the diagonal block is factored, so this file splits that loop
// into
//   diag_factor_kernel : the w x w diagonal block, one CTA, in shared memory;
//   lpanel_kernel      : rows below the block, 64 rows per CTA;
//   upanel_kernel      : columns right of the block, 64 columns per CTA;
// each replaying, per element, the reference's exact operation sequence
// (the 8-column elimination, then rank-8 updates accumulated
// acc = fma(l, u, acc) over the 8 columns and subtracted once).
// The per-element order is fixed, so results match the CPU restatement bit
// for bit.
#include "common.cuh"
#include "kernels.cuh"

namespace lub {
namespace {

constexpr int kThreads = 256;
constexpr int kStrip = 64;  // rows (lpanel) / columns (upanel) per CTA

// Factor the 8x8 tile whose rows live in lanes 0..7 of warp 0 (lane r holds
// row r in v[0..7]); tw <= 8 columns are factored.  Returns via v; writes
// 1/d into inv[].  Implements src/lu_nopiv.cu:123-171 for the tile.
__device__ __forceinline__ void factor_tile_warp(float (&v)[8], int tw,
                                                 float* inv, int64_t col0,
                                                 int* first_bad) {
  const int r = threadIdx.x & 31;
  const unsigned mask = 0xffffffffu;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    if (k < tw) {
      const float d = __shfl_sync(mask, v[k], k);
      const float iv = __fdiv_rn(1.0f, d);
      if (r == 0) {
        inv[k] = iv;
        note_pivot(d, col0 + k, first_bad);
      }
      if (r > k && r < tw) v[k] = __fmul_rn(v[k], iv);
#pragma unroll
      for (int c = k + 1; c < 8; ++c) {
        const float ukc = __shfl_sync(mask, v[c], k);
        if (c < tw && r > k && r < 8) v[c] = __fmaf_rn(-v[k], ukc, v[c]);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Diagonal block: w x w (w <= 128) at a (lda), factored in place.
// Shared: D[w x w] column-major with leading dimension LD = w | 1.
__global__ void __launch_bounds__(kThreads)
diag_factor_kernel(float* __restrict__ a, int64_t lda, int w, int64_t col0,
                   int* first_bad) {
  extern __shared__ float smem[];
  const int LD = w | 1;
  float* D = smem;
  float* inv = smem + (size_t)LD * w;
  const int tid = threadIdx.x;

  for (int idx = tid; idx < w * w; idx += kThreads) {
    const int i = idx % w, j = idx / w;
    D[i + j * LD] = a[i + (int64_t)j * lda];
  }
  __syncthreads();

  const int nt = (w + 7) / 8;
  for (int t = 0; t < nt; ++t) {
    const int t0 = 8 * t;
    const int tw = min(8, w - t0);
    // Phase A: factor the tile (warp 0, lane = tile row).
    if (tid < 32) {
      float v[8];
#pragma unroll
      for (int c = 0; c < 8; ++c)
        v[c] = (tid < tw && c < tw) ? D[(t0 + tid) + (t0 + c) * LD] : 0.0f;
      factor_tile_warp(v, tw, inv, col0 + t0, first_bad);
      if (tid < tw) {
#pragma unroll
        for (int c = 0; c < 8; ++c)
          if (c < tw) D[(t0 + tid) + (t0 + c) * LD] = v[c];
      }
    }
    __syncthreads();
    const int s = w - t0 - 8;  // trailing extent inside the block
    if (s <= 0) break;
    // Phase B: L rows below the tile (threads 0..127), U columns right of it
    // (threads 128..255).
    if (tid < 128) {
      if (tid < s) {
        const int i = t0 + 8 + tid;
        float row[8];
#pragma unroll
        for (int c = 0; c < 8; ++c) row[c] = D[i + (t0 + c) * LD];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          row[k] = __fmul_rn(row[k], inv[k]);
#pragma unroll
          for (int c = k + 1; c < 8; ++c)
            row[c] = __fmaf_rn(-row[k], D[(t0 + k) + (t0 + c) * LD], row[c]);
        }
#pragma unroll
        for (int c = 0; c < 8; ++c) D[i + (t0 + c) * LD] = row[c];
      }
    } else {
      const int q = tid - 128;
      if (q < s) {
        const int j = t0 + 8 + q;
        float col[8];
#pragma unroll
        for (int r = 0; r < 8; ++r) col[r] = D[(t0 + r) + j * LD];
#pragma unroll
        for (int k = 0; k < 8; ++k)
#pragma unroll
          for (int r = k + 1; r < 8; ++r)
            col[r] = __fmaf_rn(-D[(t0 + r) + (t0 + k) * LD], col[k], col[r]);
#pragma unroll
        for (int r = 0; r < 8; ++r) D[(t0 + r) + j * LD] = col[r];
      }
    }
    __syncthreads();
    // Phase C: rank-8 update of the trailing s x s block, 4x4 per item.
    const int nb4 = (s + 3) / 4;
    for (int b = tid; b < nb4 * nb4; b += kThreads) {
      const int i0 = t0 + 8 + 4 * (b % nb4);
      const int j0 = t0 + 8 + 4 * (b / nb4);
      float acc[4][4];
#pragma unroll
      for (int ii = 0; ii < 4; ++ii)
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) acc[ii][jj] = 0.0f;
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        float l[4], u[4];
#pragma unroll
        for (int ii = 0; ii < 4; ++ii)
          l[ii] = (i0 + ii < w) ? D[(i0 + ii) + (t0 + k) * LD] : 0.0f;
#pragma unroll
        for (int jj = 0; jj < 4; ++jj)
          u[jj] = (j0 + jj < w) ? D[(t0 + k) + (j0 + jj) * LD] : 0.0f;
#pragma unroll
        for (int ii = 0; ii < 4; ++ii)
#pragma unroll
          for (int jj = 0; jj < 4; ++jj)
            acc[ii][jj] = __fmaf_rn(l[ii], u[jj], acc[ii][jj]);
      }
#pragma unroll
      for (int ii = 0; ii < 4; ++ii)
#pragma unroll
        for (int jj = 0; jj < 4; ++jj)
          if (i0 + ii < w && j0 + jj < w) {
            float* p = &D[(i0 + ii) + (j0 + jj) * LD];
            *p = __fsub_rn(*p, acc[ii][jj]);
          }
    }
    __syncthreads();
  }

  for (int idx = tid; idx < w * w; idx += kThreads) {
    const int i = idx % w, j = idx / w;
    a[i + (int64_t)j * lda] = D[i + j * LD];
  }
}

// ---------------------------------------------------------------------------
// L panel: rows [0, M) of `a` (lda) with w columns, against the factored
// diagonal block `dg` (lda), in place.
__global__ void __launch_bounds__(kThreads)
lpanel_kernel(float* __restrict__ a, int64_t lda, const float* __restrict__ dg,
              int64_t M, int w) {
  extern __shared__ float smem[];
  constexpr int LDS = kStrip + 1;
  float* S = smem;                       // kStrip x w, column-major, ld LDS
  float* Ut = S + (size_t)LDS * w;       // 8 x w, row-major (Ut[k*w + c])
  float* inv = Ut + 8 * w;               // 8
  const int tid = threadIdx.x;
  const int64_t r0 = (int64_t)blockIdx.x * kStrip;
  const int rows = (int)((M - r0) < kStrip ? (M - r0) : kStrip);

  for (int idx = tid; idx < kStrip * w; idx += kThreads) {
    const int i = idx % kStrip, j = idx / kStrip;
    S[i + j * LDS] = (i < rows) ? a[(r0 + i) + (int64_t)j * lda] : 0.0f;
  }

  const int nt = (w + 7) / 8;
  for (int t = 0; t < nt; ++t) {
    const int t0 = 8 * t;
    const int tw = min(8, w - t0);
    __syncthreads();  // previous phase done with Ut / S
    for (int idx = tid; idx < 8 * (w - t0); idx += kThreads) {
      const int k = idx / (w - t0), c = t0 + idx % (w - t0);
      Ut[k * w + c] = (k < tw) ? dg[(t0 + k) + (int64_t)c * lda] : 0.0f;
    }
    if (tid < 8) inv[tid] = (tid < tw) ? __fdiv_rn(1.0f, dg[(t0 + tid) + (int64_t)(t0 + tid) * lda]) : 0.0f;
    __syncthreads();
    // Phase A: eliminate the tile columns of each row.
    if (tid < kStrip) {
      float row[8];
#pragma unroll
      for (int c = 0; c < 8; ++c) row[c] = (c < tw) ? S[tid + (t0 + c) * LDS] : 0.0f;
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        if (k < tw) {
          row[k] = __fmul_rn(row[k], inv[k]);
#pragma unroll
          for (int c = k + 1; c < 8; ++c)
            if (c < tw) row[c] = __fmaf_rn(-row[k], Ut[k * w + t0 + c], row[c]);
        }
      }
#pragma unroll
      for (int c = 0; c < 8; ++c)
        if (c < tw) S[tid + (t0 + c) * LDS] = row[c];
    }
    const int s = w - t0 - 8;
    if (s <= 0) break;
    __syncthreads();
    // Phase B: rank-8 update of the trailing columns (4 rows x 4 cols/item).
    const int ncb = (s + 3) / 4;
    for (int b = tid; b < (kStrip / 4) * ncb; b += kThreads) {
      const int i0 = 4 * (b % (kStrip / 4));
      const int c0 = t0 + 8 + 4 * (b / (kStrip / 4));
      float acc[4][4];
#pragma unroll
      for (int ii = 0; ii < 4; ++ii)
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) acc[ii][jj] = 0.0f;
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        float l[4], u[4];
#pragma unroll
        for (int ii = 0; ii < 4; ++ii) l[ii] = S[(i0 + ii) + (t0 + k) * LDS];
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) u[jj] = (c0 + jj < w) ? Ut[k * w + c0 + jj] : 0.0f;
#pragma unroll
        for (int ii = 0; ii < 4; ++ii)
#pragma unroll
          for (int jj = 0; jj < 4; ++jj)
            acc[ii][jj] = __fmaf_rn(l[ii], u[jj], acc[ii][jj]);
      }
#pragma unroll
      for (int ii = 0; ii < 4; ++ii)
#pragma unroll
        for (int jj = 0; jj < 4; ++jj)
          if (c0 + jj < w) {
            float* p = &S[(i0 + ii) + (c0 + jj) * LDS];
            *p = __fsub_rn(*p, acc[ii][jj]);
          }
    }
  }
  __syncthreads();
  for (int idx = tid; idx < kStrip * w; idx += kThreads) {
    const int i = idx % kStrip, j = idx / kStrip;
    if (i < rows) a[(r0 + i) + (int64_t)j * lda] = S[i + j * LDS];
  }
}

// ---------------------------------------------------------------------------
// U panel: w rows of the block row starting at `a` (lda), columns [0, N),
// against the factored diagonal block `dg` (lda), in place.
__global__ void __launch_bounds__(kThreads)
upanel_kernel(float* __restrict__ a, int64_t lda, const float* __restrict__ dg,
              int64_t N, int w) {
  extern __shared__ float smem[];
  const int LDS = w | 1;
  float* S = smem;                    // w x kStrip, column-major, ld LDS
  float* Lt = S + (size_t)LDS * kStrip;  // w x 8, Lt[r*8 + k]
  const int tid = threadIdx.x;
  const int64_t c0g = (int64_t)blockIdx.x * kStrip;
  const int cols = (int)((N - c0g) < kStrip ? (N - c0g) : kStrip);

  for (int idx = tid; idx < kStrip * w; idx += kThreads) {
    const int i = idx % w, j = idx / w;
    S[i + j * LDS] = (j < cols) ? a[i + (c0g + j) * lda] : 0.0f;
  }

  const int nt = (w + 7) / 8;
  for (int t = 0; t < nt; ++t) {
    const int t0 = 8 * t;
    const int tw = min(8, w - t0);
    __syncthreads();
    for (int idx = tid; idx < 8 * (w - t0); idx += kThreads) {
      const int k = idx % 8, r = t0 + idx / 8;
      Lt[r * 8 + k] = (k < tw) ? dg[r + (int64_t)(t0 + k) * lda] : 0.0f;
    }
    __syncthreads();
    // Phase A: forward substitution with the unit-lower tile.
    if (tid < kStrip) {
      float col[8];
#pragma unroll
      for (int r = 0; r < 8; ++r) col[r] = (r < tw) ? S[(t0 + r) + tid * LDS] : 0.0f;
#pragma unroll
      for (int k = 0; k < 8; ++k)
#pragma unroll
        for (int r = k + 1; r < 8; ++r)
          if (k < tw && r < tw)
            col[r] = __fmaf_rn(-Lt[(t0 + r) * 8 + k], col[k], col[r]);
#pragma unroll
      for (int r = 0; r < 8; ++r)
        if (r < tw) S[(t0 + r) + tid * LDS] = col[r];
    }
    const int s = w - t0 - 8;
    if (s <= 0) break;
    __syncthreads();
    // Phase B: rank-8 update of the remaining rows (4 rows x 4 cols/item).
    const int nrb = (s + 3) / 4;
    for (int b = tid; b < nrb * (kStrip / 4); b += kThreads) {
      const int i0 = t0 + 8 + 4 * (b % nrb);
      const int j0 = 4 * (b / nrb);
      float acc[4][4];
#pragma unroll
      for (int ii = 0; ii < 4; ++ii)
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) acc[ii][jj] = 0.0f;
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        float l[4], u[4];
#pragma unroll
        for (int ii = 0; ii < 4; ++ii) l[ii] = (i0 + ii < w) ? Lt[(i0 + ii) * 8 + k] : 0.0f;
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) u[jj] = S[(t0 + k) + (j0 + jj) * LDS];
#pragma unroll
        for (int ii = 0; ii < 4; ++ii)
#pragma unroll
          for (int jj = 0; jj < 4; ++jj)
            acc[ii][jj] = __fmaf_rn(l[ii], u[jj], acc[ii][jj]);
      }
#pragma unroll
      for (int ii = 0; ii < 4; ++ii)
#pragma unroll
        for (int jj = 0; jj < 4; ++jj)
          if (i0 + ii < w) {
            float* p = &S[(i0 + ii) + (j0 + jj) * LDS];
            *p = __fsub_rn(*p, acc[ii][jj]);
          }
    }
  }
  __syncthreads();
  for (int idx = tid; idx < kStrip * w; idx += kThreads) {
    const int i = idx % w, j = idx / w;
    if (j < cols) a[i + (c0g + j) * lda] = S[i + j * LDS];
  }
}

// ---------------------------------------------------------------------------
// Reference-compatible panel (remifa::lu_nopiv_panel<float,8>): n <= 8
// columns, the diagonal tile factored from the copy d by every CTA.
// blockIdx.y == 0: L rows [n, m); blockIdx.y == 1: U columns [n, m).
__global__ void __launch_bounds__(kThreads)
ref_panel_kernel(int64_t m, int n, const float* __restrict__ d, int64_t ldd,
                 float* __restrict__ l, int64_t ldl, float* __restrict__ u,
                 int64_t ldu, int* stat) {
  __shared__ float T[8][9];
  __shared__ float inv[8];
  const int tid = threadIdx.x;
  if (tid < 32) {
    float v[8];
#pragma unroll
    for (int c = 0; c < 8; ++c)
      v[c] = (tid < n && c < n) ? d[tid + c * ldd] : 0.0f;
    factor_tile_warp(v, n, inv, 0, nullptr);
    if (tid < 8) {
#pragma unroll
      for (int c = 0; c < 8; ++c) T[tid][c] = v[c];
    }
  }
  __syncthreads();
  if (blockIdx.x == 0 && blockIdx.y == 0) {
    if (tid < 64) {
      const int r = tid % 8, c = tid / 8;
      if (r < n && c < n) l[r + c * ldl] = T[r][c];
    }
    if (tid == 0 && stat) *stat = n;
  }
  const int64_t q = (int64_t)blockIdx.x * kThreads + tid + n;
  if (q >= m) return;
  if (blockIdx.y == 0) {
    float row[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) row[c] = (c < n) ? l[q + c * ldl] : 0.0f;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      if (k < n) {
        row[k] = __fmul_rn(row[k], inv[k]);
#pragma unroll
        for (int c = k + 1; c < 8; ++c)
          if (c < n) row[c] = __fmaf_rn(-row[k], T[k][c], row[c]);
      }
    }
#pragma unroll
    for (int c = 0; c < 8; ++c)
      if (c < n) l[q + c * ldl] = row[c];
  } else {
    float col[8];
#pragma unroll
    for (int r = 0; r < 8; ++r) col[r] = (r < n) ? u[r + q * ldu] : 0.0f;
#pragma unroll
    for (int k = 0; k < 8; ++k)
#pragma unroll
      for (int r = k + 1; r < 8; ++r)
        if (k < n && r < n) col[r] = __fmaf_rn(-T[r][k], col[k], col[r]);
#pragma unroll
    for (int r = 0; r < 8; ++r)
      if (r < n) u[r + q * ldu] = col[r];
  }
}

}  // namespace

// ---------------------------------------------------------------------------
// launchers

size_t diag_smem_bytes(int w) {
  return ((size_t)(w | 1) * w + 8) * sizeof(float);
}

lu_status launch_diag_factor(cudaStream_t st, float* a, int64_t lda, int w,
                             int64_t col0, int* first_bad) {
  if (w <= 0 || w > 128) return LU_ERR_INVALID_ARG;
  const size_t sm = diag_smem_bytes(w);
  LUB_CUDA_TRY(set_smem_limit((const void*)diag_factor_kernel, sm));
  diag_factor_kernel<<<1, kThreads, sm, st>>>(a, lda, w, col0, first_bad);
  LUB_LAUNCH_CHECK();
  return LU_SUCCESS;
}

lu_status launch_lpanel(cudaStream_t st, float* a, int64_t lda, const float* dg,
                        int64_t M, int w) {
  if (M <= 0) return LU_SUCCESS;
  if (w <= 0 || w > 256) return LU_ERR_INVALID_ARG;
  const size_t sm = ((size_t)(kStrip + 1) * w + 8 * (size_t)w + 8) * sizeof(float);
  LUB_CUDA_TRY(set_smem_limit((const void*)lpanel_kernel, sm));
  const int64_t grid = ceil_div(M, kStrip);
  lpanel_kernel<<<(unsigned)grid, kThreads, sm, st>>>(a, lda, dg, M, w);
  LUB_LAUNCH_CHECK();
  return LU_SUCCESS;
}

lu_status launch_upanel(cudaStream_t st, float* a, int64_t lda, const float* dg,
                        int64_t N, int w) {
  if (N <= 0) return LU_SUCCESS;
  if (w <= 0 || w > 256) return LU_ERR_INVALID_ARG;
  const size_t sm = ((size_t)(w | 1) * kStrip + 8 * (size_t)w) * sizeof(float);
  LUB_CUDA_TRY(set_smem_limit((const void*)upanel_kernel, sm));
  const int64_t grid = ceil_div(N, kStrip);
  upanel_kernel<<<(unsigned)grid, kThreads, sm, st>>>(a, lda, dg, N, w);
  LUB_LAUNCH_CHECK();
  return LU_SUCCESS;
}

lu_status launch_ref_panel(cudaStream_t st, int64_t m, int n, const float* d,
                           int64_t ldd, float* l, int64_t ldl, float* u,
                           int64_t ldu, int* stat) {
  if (n <= 0 || n > 8 || m < n) return LU_ERR_INVALID_ARG;
  const int64_t rest = m - n;
  dim3 grid((unsigned)std::max<int64_t>(1, ceil_div(rest, kThreads)), 2);
  ref_panel_kernel<<<grid, kThreads, 0, st>>>(m, n, d, ldd, l, ldl, u, ldu, stat);
  LUB_LAUNCH_CHECK();
  return LU_SUCCESS;
}

}  // namespace lub
