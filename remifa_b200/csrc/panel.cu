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
// Diagonal block: w x w (w <= 128) at a (lda), factored in place by one CTA.
// Shared: D (w x w, column-major, leading dimension LD = round4(w) + 4 so
// 4-row groups are 16-byte aligned), plus the L and U strips of the current
// tile (Ls[k][i], Us[k][j]) for vectorised rank-8 updates.
__global__ void __launch_bounds__(kThreads)
diag_factor_kernel(float* __restrict__ a, int64_t lda, int w, int64_t col0,
                   int* first_bad) {
  extern __shared__ __align__(16) float smem[];
  const int LD = ((w + 3) / 4) * 4 + 4;
  float* D = smem;
  float* Ls = D + (size_t)LD * w;     // [8][128]
  float* Us = Ls + 8 * 128;           // [8][128]
  float* inv = Us + 8 * 128;          // [8]
  const int tid = threadIdx.x;

  for (int idx = tid; idx < w * w; idx += kThreads) {
    const int i = idx % w, j = idx / w;
    cp_async4(&D[i + j * LD], &a[i + (int64_t)j * lda]);
  }
  cp_async_wait_all();
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
    // (threads 128..255); results also go to the strip buffers.
    if (tid < 128) {
      if (tid < s) {
        const int i = t0 + 8 + tid;
        float u[8][8];
#pragma unroll
        for (int k = 0; k < 8; ++k)
#pragma unroll
          for (int c = k + 1; c < 8; ++c) u[k][c] = D[(t0 + k) + (t0 + c) * LD];
        float row[8];
#pragma unroll
        for (int c = 0; c < 8; ++c) row[c] = D[i + (t0 + c) * LD];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          row[k] = __fmul_rn(row[k], inv[k]);
#pragma unroll
          for (int c = k + 1; c < 8; ++c) row[c] = __fmaf_rn(-row[k], u[k][c], row[c]);
        }
#pragma unroll
        for (int c = 0; c < 8; ++c) {
          D[i + (t0 + c) * LD] = row[c];
          Ls[c * 128 + (i - t0 - 8)] = row[c];
        }
      }
    } else {
      const int q = tid - 128;
      if (q < s) {
        const int j = t0 + 8 + q;
        float l[8][8];
#pragma unroll
        for (int k = 0; k < 8; ++k)
#pragma unroll
          for (int r = k + 1; r < 8; ++r) l[r][k] = D[(t0 + r) + (t0 + k) * LD];
        float col[8];
#pragma unroll
        for (int r = 0; r < 8; ++r) col[r] = D[(t0 + r) + j * LD];
#pragma unroll
        for (int k = 0; k < 8; ++k)
#pragma unroll
          for (int r = k + 1; r < 8; ++r) col[r] = __fmaf_rn(-l[r][k], col[k], col[r]);
#pragma unroll
        for (int r = 0; r < 8; ++r) {
          D[(t0 + r) + j * LD] = col[r];
          Us[r * 128 + q] = col[r];
        }
      }
    }
    __syncthreads();
    // Phase C: rank-8 update of the trailing s x s block, 4 x 4 per item:
    // acc = sum_k fma(L[i][t0+k], U[t0+k][j]) in k order, D[i][j] -= acc.
    const int nb4 = (s + 3) / 4;
    const bool vec = (s % 4 == 0);
    for (int b = tid; b < nb4 * nb4; b += kThreads) {
      const int li = 4 * (b % nb4), lj = 4 * (b / nb4);  // local to the block
      const int i0 = t0 + 8 + li, j0 = t0 + 8 + lj;
      float acc[4][4];
#pragma unroll
      for (int ii = 0; ii < 4; ++ii)
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) acc[ii][jj] = 0.0f;
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const float4 l4 = *reinterpret_cast<const float4*>(&Ls[k * 128 + li]);
        const float4 u4 = *reinterpret_cast<const float4*>(&Us[k * 128 + lj]);
        const float l[4] = {l4.x, l4.y, l4.z, l4.w};
        const float u[4] = {u4.x, u4.y, u4.z, u4.w};
#pragma unroll
        for (int ii = 0; ii < 4; ++ii)
#pragma unroll
          for (int jj = 0; jj < 4; ++jj)
            acc[ii][jj] = __fmaf_rn(l[ii], u[jj], acc[ii][jj]);
      }
      if (vec && (i0 % 4) == 0) {
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) {
          float4* p = reinterpret_cast<float4*>(&D[i0 + (j0 + jj) * LD]);
          float4 c4 = *p;
          c4.x = __fsub_rn(c4.x, acc[0][jj]);
          c4.y = __fsub_rn(c4.y, acc[1][jj]);
          c4.z = __fsub_rn(c4.z, acc[2][jj]);
          c4.w = __fsub_rn(c4.w, acc[3][jj]);
          *p = c4;
        }
      } else {
#pragma unroll
        for (int ii = 0; ii < 4; ++ii)
#pragma unroll
          for (int jj = 0; jj < 4; ++jj)
            if (i0 + ii < w && j0 + jj < w) {
              float* p = &D[(i0 + ii) + (j0 + jj) * LD];
              *p = __fsub_rn(*p, acc[ii][jj]);
            }
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
// L and U panels of one sub-panel, one launch.  `dg` is the factored w x w
// diagonal block (lda); M rows lie below it, N columns right of it.
// Blocks [0, nL) each own kPanelT rows of L21 (one row per thread); blocks
// [nL, ...) each own kPanelT columns of U12 (one column per thread).
// A thread walks its row (column) tile by tile, left to right: it first
// applies the rank-8 updates of all earlier tiles in order (acc over the 8
// columns, one subtraction per tile -- the sequence the reference's K = 8
// GEMMs produce), then the tile elimination of the panel kernel.  Rows and
// columns are independent, so no block-wide synchronisation is needed after
// the staging of the diagonal block.
constexpr int kPanelT = 256;

__global__ void __launch_bounds__(kPanelT)
lupanel_kernel(float* __restrict__ dg, int64_t lda, int w, int64_t M,
               int64_t N, int nL) {
  extern __shared__ __align__(16) float smem[];
  const int tid = threadIdx.x;
  const int wp = ((w + 7) / 8) * 8;  // padded width (zero filled)
  const int nt = wp / 8;
  // F[c*wp + r] = D[r][c]: the factored block, column-major with a padded
  // (zero-filled) leading dimension so 4-element groups are 16-byte aligned.
  // The L role reads its strict upper part (U), the U role its strict lower
  // part (L); the diagonal gives 1/d.
  float* F = smem;
  float* inv = F + (size_t)wp * wp;  // wp
  float* S = inv + wp;               // the strip
  const bool is_l = (int)blockIdx.x < nL;

  for (int idx = tid; idx < wp * wp; idx += kPanelT) {
    const int r = idx % wp, c = idx / wp;
    if (r < w && c < w) cp_async4(&F[idx], &dg[r + (int64_t)c * lda]);
    else F[idx] = 0.0f;
  }

  if (is_l) {
    // strip: kPanelT rows x w columns, S[c*kPanelT + r]
    const int64_t r0 = (int64_t)blockIdx.x * kPanelT;
    float* A = dg + w;  // first row below the diagonal block
    const int64_t row = r0 + tid;
    for (int c = 0; c < w; ++c) {
      if (row < M) cp_async4(&S[c * kPanelT + tid], &A[row + (int64_t)c * lda]);
      else S[c * kPanelT + tid] = 0.0f;
    }
    cp_async_wait_all();
    __syncthreads();
    for (int k = tid; k < wp; k += kPanelT)
      inv[k] = (k < w) ? __fdiv_rn(1.0f, F[k * wp + k]) : 0.0f;
    __syncthreads();
    const int r = tid;
    for (int T = 0; T < nt; ++T) {
      const int tw = min(8, w - 8 * T);
      float x[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) x[j] = (j < tw) ? S[(8 * T + j) * kPanelT + r] : 0.0f;
      for (int t = 0; t < T; ++t) {
        float acc[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[j] = 0.0f;
        float l[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) l[k] = S[(8 * t + k) * kPanelT + r];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          // U[8t .. 8t+7][8T + j]: one column of F, 8 consecutive rows
          const float4 u0 = *reinterpret_cast<const float4*>(&F[(8 * T + j) * wp + 8 * t]);
          const float4 u1 = *reinterpret_cast<const float4*>(&F[(8 * T + j) * wp + 8 * t + 4]);
          float a = acc[j];
          a = __fmaf_rn(l[0], u0.x, a);
          a = __fmaf_rn(l[1], u0.y, a);
          a = __fmaf_rn(l[2], u0.z, a);
          a = __fmaf_rn(l[3], u0.w, a);
          a = __fmaf_rn(l[4], u1.x, a);
          a = __fmaf_rn(l[5], u1.y, a);
          a = __fmaf_rn(l[6], u1.z, a);
          a = __fmaf_rn(l[7], u1.w, a);
          acc[j] = a;
        }
#pragma unroll
        for (int j = 0; j < 8; ++j) x[j] = __fsub_rn(x[j], acc[j]);
      }
      // tile elimination (src/lu_nopiv.cu:141-168): 1/d multiply, fused
      // rank-1 updates inside the tile
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        if (k < tw) {
          x[k] = __fmul_rn(x[k], inv[8 * T + k]);
#pragma unroll
          for (int j = k + 1; j < 8; ++j)
            if (j < tw) x[j] = __fmaf_rn(-x[k], F[(8 * T + j) * wp + 8 * T + k], x[j]);
        }
      }
#pragma unroll
      for (int j = 0; j < 8; ++j)
        if (j < tw) S[(8 * T + j) * kPanelT + r] = x[j];
    }
    for (int c = 0; c < w; ++c)
      if (row < M) A[row + (int64_t)c * lda] = S[c * kPanelT + tid];
  } else {
    // strip: w rows x kPanelT columns, S[i*(kPanelT+1) + c]
    constexpr int LS = kPanelT + 1;
    const int64_t c0 = (int64_t)(blockIdx.x - nL) * kPanelT;
    float* A = dg + (int64_t)w * lda;  // first column right of the block
    for (int idx = tid; idx < w * kPanelT; idx += kPanelT) {
      const int i = idx % w, cc = idx / w;
      const int64_t col = c0 + cc;
      if (col < N) cp_async4(&S[i * LS + cc], &A[i + col * lda]);
      else S[i * LS + cc] = 0.0f;
    }
    cp_async_wait_all();
    __syncthreads();
    const int c = tid;
    for (int T = 0; T < nt; ++T) {
      const int tw = min(8, w - 8 * T);
      float x[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) x[j] = (j < tw) ? S[(8 * T + j) * LS + c] : 0.0f;
      for (int t = 0; t < T; ++t) {
        float acc[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[j] = 0.0f;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          const float u = S[(8 * t + k) * LS + c];
          const float4 l0 = *reinterpret_cast<const float4*>(&F[(8 * t + k) * wp + 8 * T]);
          const float4 l1 = *reinterpret_cast<const float4*>(&F[(8 * t + k) * wp + 8 * T + 4]);
          acc[0] = __fmaf_rn(l0.x, u, acc[0]);
          acc[1] = __fmaf_rn(l0.y, u, acc[1]);
          acc[2] = __fmaf_rn(l0.z, u, acc[2]);
          acc[3] = __fmaf_rn(l0.w, u, acc[3]);
          acc[4] = __fmaf_rn(l1.x, u, acc[4]);
          acc[5] = __fmaf_rn(l1.y, u, acc[5]);
          acc[6] = __fmaf_rn(l1.z, u, acc[6]);
          acc[7] = __fmaf_rn(l1.w, u, acc[7]);
        }
#pragma unroll
        for (int j = 0; j < 8; ++j) x[j] = __fsub_rn(x[j], acc[j]);
      }
      // forward substitution with the unit-lower tile (src/lu_nopiv.cu:304-316)
#pragma unroll
      for (int k = 0; k < 8; ++k)
#pragma unroll
        for (int j = k + 1; j < 8; ++j)
          if (k < tw && j < tw)
            x[j] = __fmaf_rn(-F[(8 * T + k) * wp + 8 * T + j], x[k], x[j]);
#pragma unroll
      for (int j = 0; j < 8; ++j)
        if (j < tw) S[(8 * T + j) * LS + c] = x[j];
    }
    __syncthreads();
    for (int idx = tid; idx < w * kPanelT; idx += kPanelT) {
      const int i = idx % w, cc = idx / w;
      const int64_t col = c0 + cc;
      if (col < N) A[i + col * lda] = S[i * LS + cc];
    }
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
  const int LD = ((w + 3) / 4) * 4 + 4;
  return ((size_t)LD * w + 2 * 8 * 128 + 8) * sizeof(float);
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

static size_t lupanel_smem_bytes(int w) {
  const size_t wp = (size_t)((w + 7) / 8) * 8;
  const size_t strip = std::max<size_t>((size_t)kPanelT * wp, wp * (kPanelT + 1));
  return (wp * wp + wp + strip) * sizeof(float);
}

lu_status launch_lupanel(cudaStream_t st, float* dg, int64_t lda, int w,
                         int64_t M, int64_t N) {
  if (w <= 0 || w > 128) return LU_ERR_INVALID_ARG;
  const int64_t nL = M > 0 ? ceil_div(M, kPanelT) : 0;
  const int64_t nU = N > 0 ? ceil_div(N, kPanelT) : 0;
  if (nL + nU == 0) return LU_SUCCESS;
  const size_t sm = lupanel_smem_bytes(w);
  LUB_CUDA_TRY(set_smem_limit((const void*)lupanel_kernel, sm));
  lupanel_kernel<<<(unsigned)(nL + nU), kPanelT, sm, st>>>(dg, lda, w, M, N, (int)nL);
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
