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
      const float iv = __frcp_rn(d);  // correctly rounded 1/d
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

// The same tile factorization by a single thread, the tile held in
// registers (T points at its top-left element in shared memory, ld LD).
__device__ __forceinline__ void factor_tile_thread(float* T, int LD, int tw,
                                                   float* inv, int64_t col0,
                                                   int* first_bad) {
  float v[8][8];
#pragma unroll
  for (int r = 0; r < 8; ++r)
#pragma unroll
    for (int c = 0; c < 8; ++c) v[r][c] = (r < tw && c < tw) ? T[r + c * LD] : 0.0f;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    if (k < tw) {
      const float d = v[k][k];
      note_pivot(d, col0 + k, first_bad);
      const float iv = __frcp_rn(d);  // correctly rounded 1/d
      inv[k] = iv;
#pragma unroll
      for (int r = k + 1; r < 8; ++r) v[r][k] = __fmul_rn(v[r][k], iv);
#pragma unroll
      for (int c = k + 1; c < 8; ++c)
#pragma unroll
        for (int r = k + 1; r < 8; ++r) v[r][c] = __fmaf_rn(-v[r][k], v[k][c], v[r][c]);
    }
  }
#pragma unroll
  for (int r = 0; r < 8; ++r)
#pragma unroll
    for (int c = 0; c < 8; ++c)
      if (r < tw && c < tw) T[r + c * LD] = v[r][c];
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
    // Phase A: one thread factors the 8 x 8 tile in registers
    // (src/lu_nopiv.cu:123-171): 1/d, scale the column below, fused rank-1
    // update of the rest of the tile.
    if (tid == 0) factor_tile_thread(D + t0 + t0 * LD, LD, tw, inv, col0 + t0, first_bad);
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
// Diagonal block of the left-looking (Crout) variant, w <= 128, one CTA.
// Per tile T, in the reference's order (src/lu_nopiv_inner_ll.hxx:197-370):
// the tile column (rows >= 8T) and the tile row (columns right of the tile)
// receive one update summing all earlier columns of the block (acc over
// k < 8T, subtracted once), then the tile is factored and the L rows and U
// columns of the block are eliminated with it.
__global__ void __launch_bounds__(kThreads)
diag_crout_kernel(float* __restrict__ a, int64_t lda, int w, int64_t col0,
                  int* first_bad) {
  extern __shared__ __align__(16) float smem[];
  const int LD = ((w + 3) / 4) * 4 + 4;
  float* D = smem;
  float* inv = D + (size_t)LD * w;  // 8
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
    if (t0 > 0) {
      // (a) tile column: rows [t0, w) x cols [t0, t0+tw); tile row: rows
      // [t0, t0+tw) x cols [t0+tw, w)
      const int ncol = (w - t0) * tw;
      const int nrow = tw * (w - t0 - tw);
      for (int e = tid; e < ncol + nrow; e += kThreads) {
        int i, c;
        if (e < ncol) { i = t0 + e % (w - t0); c = t0 + e / (w - t0); }
        else { const int f = e - ncol; i = t0 + f % tw; c = t0 + tw + f / tw; }
        float acc = 0.0f;
        for (int k = 0; k < t0; ++k) acc = __fmaf_rn(D[i + k * LD], D[k + c * LD], acc);
        D[i + c * LD] = __fsub_rn(D[i + c * LD], acc);
      }
      __syncthreads();
    }
    // (b) factor the tile
    if (tid == 0) factor_tile_thread(D + t0 + t0 * LD, LD, tw, inv, col0 + t0, first_bad);
    __syncthreads();
    const int s = w - t0 - tw;
    if (s <= 0) break;
    // (c) eliminate the block's L rows / U columns with the tile
    if (tid < 128) {
      if (tid < s) {
        const int i = t0 + tw + tid;
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
        const int j = t0 + tw + q;
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
  }
  for (int idx = tid; idx < w * w; idx += kThreads) {
    const int i = idx % w, j = idx / w;
    a[i + (int64_t)j * lda] = D[i + j * LD];
  }
}

// ---------------------------------------------------------------------------
// L and U panels of one sub-panel, one launch.  `dg` is the factored w x w
// diagonal block (lda); M rows lie below it, N columns right of it.
//
// Eight threads (one group, lane & 7 = j) own one row of L21 (L blocks) or
// one column of U12 (U blocks); a CTA of 256 threads owns 32 of them.  The
// group walks its row (column) tile by tile, left to right.  For tile T,
// thread j first applies the rank-8 updates of all earlier tiles to element
// j of the tile, in order (acc = sum over the 8 columns of the earlier tile
// with fused multiply-adds, then one subtraction per tile: the sequence the
// reference's K = 8 GEMMs produce), then the group performs the tile
// elimination of the panel kernel, passing the eliminated value of column k
// to the others with a shuffle.  Rows (columns) are independent, so the
// only synchronisation after staging is within the 8-lane group.
constexpr int kPanelT = 256;
constexpr int kGroup = 8;
constexpr int kItems = kPanelT / kGroup;  // rows / columns per CTA

__global__ void __launch_bounds__(kPanelT)
lupanel_kernel(float* __restrict__ dg, int64_t lda, int w, int64_t M,
               int64_t N, int nL, bool left) {
  extern __shared__ __align__(16) float smem[];
  const int tid = threadIdx.x;
  const int wp = ((w + 7) / 8) * 8;  // padded width (zero filled)
  const int nt = wp / 8;
  const int ls = wp + 4;             // strip row stride (breaks bank aliasing)
  const int lf = wp + 4;             // leading dimension of F, same reason
  float* F = smem;                   // diagonal block, wp x wp, F[c*lf + r]
  float* inv = F + (size_t)wp * lf;  // wp
  float* S = inv + wp;               // kItems x ls
  const bool is_l = (int)blockIdx.x < nL;
  const int j = tid & (kGroup - 1);
  const int q = tid / kGroup;        // item of this group
  const unsigned gmask = 0xffu << (tid & 24);  // the 8 lanes of the group

  // Stage the factored diagonal block, column-major with a padded leading
  // dimension (F[c*lf + r] = D[r][c]): U[8t..8t+7][c] is one aligned 8-float
  // run, and the 8 columns a group reads at once fall in distinct banks.
  for (int idx = tid; idx < wp * wp; idx += kPanelT) {
    const int r = idx % wp, c = idx / wp;
    if (r < w && c < w) cp_async4(&F[c * lf + r], &dg[r + (int64_t)c * lda]);
    else F[c * lf + r] = 0.0f;
  }
  int64_t item0;
  float* A;
  int64_t count;
  if (is_l) {
    item0 = (int64_t)blockIdx.x * kItems;
    A = dg + w;                      // first row below the block
    count = M;
    // strip: S[q*ls + c] = A[row q, column c]; consecutive threads read
    // consecutive rows of one column
    for (int idx = tid; idx < kItems * wp; idx += kPanelT) {
      const int qq = idx % kItems, c = idx / kItems;
      const int64_t row = item0 + qq;
      if (row < M && c < w) cp_async4(&S[qq * ls + c], &A[row + (int64_t)c * lda]);
      else S[qq * ls + c] = 0.0f;
    }
  } else {
    item0 = (int64_t)(blockIdx.x - nL) * kItems;
    A = dg + (int64_t)w * lda;       // first column right of the block
    count = N;
    // strip: S[q*ls + i] = A[row i, column q]; consecutive threads read
    // consecutive rows of one column
    for (int idx = tid; idx < kItems * wp; idx += kPanelT) {
      const int i = idx % wp, qq = idx / wp;
      const int64_t col = item0 + qq;
      if (col < N && i < w) cp_async4(&S[qq * ls + i], &A[i + col * lda]);
      else S[qq * ls + i] = 0.0f;
    }
  }
  cp_async_wait_all();
  __syncthreads();
  if (is_l) {
    for (int k = tid; k < wp; k += kPanelT)
      inv[k] = (k < w) ? __frcp_rn(F[k * lf + k]) : 0.0f;
    __syncthreads();
  }

  const bool valid = item0 + q < count;
  float* srow = S + q * ls;
  for (int T = 0; T < nt; ++T) {
    const int tw = min(8, w - 8 * T);
    float x = srow[8 * T + j];
    // updates of earlier tiles, in order.  Right-looking (the reference's
    // lu_nopiv_inner_rl): one subtraction per earlier tile.  Left-looking
    // (lu_nopiv_inner_ll, src/lu_nopiv_inner_ll.hxx:225-300): one sum over
    // all earlier columns, subtracted once.
    float accl = 0.0f;
    for (int t = 0; t < T; ++t) {
      const float4 v0 = *reinterpret_cast<const float4*>(&srow[8 * t]);
      const float4 v1 = *reinterpret_cast<const float4*>(&srow[8 * t + 4]);
      float acc = left ? accl : 0.0f;
      if (is_l) {
        // U[8t+k][8T+j]: column 8T+j of F, rows 8t..8t+7
        const float* fcol = &F[(8 * T + j) * lf + 8 * t];
        const float4 f0 = *reinterpret_cast<const float4*>(fcol);
        const float4 f1 = *reinterpret_cast<const float4*>(fcol + 4);
        acc = __fmaf_rn(v0.x, f0.x, acc);
        acc = __fmaf_rn(v0.y, f0.y, acc);
        acc = __fmaf_rn(v0.z, f0.z, acc);
        acc = __fmaf_rn(v0.w, f0.w, acc);
        acc = __fmaf_rn(v1.x, f1.x, acc);
        acc = __fmaf_rn(v1.y, f1.y, acc);
        acc = __fmaf_rn(v1.z, f1.z, acc);
        acc = __fmaf_rn(v1.w, f1.w, acc);
      } else {
        // L[8T+j][8t+k]: row 8T+j of F, columns 8t..8t+7 (the 8 lanes of a
        // group read 8 consecutive words)
        const float* frow = &F[(8 * t) * lf + 8 * T + j];
        acc = __fmaf_rn(frow[0 * lf], v0.x, acc);
        acc = __fmaf_rn(frow[1 * lf], v0.y, acc);
        acc = __fmaf_rn(frow[2 * lf], v0.z, acc);
        acc = __fmaf_rn(frow[3 * lf], v0.w, acc);
        acc = __fmaf_rn(frow[4 * lf], v1.x, acc);
        acc = __fmaf_rn(frow[5 * lf], v1.y, acc);
        acc = __fmaf_rn(frow[6 * lf], v1.z, acc);
        acc = __fmaf_rn(frow[7 * lf], v1.w, acc);
      }
      if (left) accl = acc;
      else x = __fsub_rn(x, acc);
    }
    if (left && T > 0) x = __fsub_rn(x, accl);
    // tile elimination
    if (is_l) {
      // src/lu_nopiv.cu:141-168: x_k *= 1/d_k, then x_j -= x_k * U[k][j]
      for (int k = 0; k < tw; ++k) {
        if (j == k) x = __fmul_rn(x, inv[8 * T + k]);
        const float xk = __shfl_sync(gmask, x, k, kGroup);
        if (j > k && j < tw) x = __fmaf_rn(-xk, F[(8 * T + j) * lf + 8 * T + k], x);
      }
    } else {
      // src/lu_nopiv.cu:304-316: x_j -= L[j][k] * x_k (unit diagonal)
      for (int k = 0; k < tw; ++k) {
        const float xk = __shfl_sync(gmask, x, k, kGroup);
        if (j > k && j < tw) x = __fmaf_rn(-F[(8 * T + k) * lf + 8 * T + j], xk, x);
      }
    }
    if (j < tw) srow[8 * T + j] = x;
    __syncwarp(gmask);
  }
  __syncthreads();
  if (is_l) {
    for (int idx = tid; idx < kItems * w; idx += kPanelT) {
      const int qq = idx % kItems, c = idx / kItems;
      const int64_t row = item0 + qq;
      if (row < M) A[row + (int64_t)c * lda] = S[qq * ls + c];
    }
  } else {
    for (int idx = tid; idx < kItems * w; idx += kPanelT) {
      const int i = idx % w, qq = idx / w;
      const int64_t col = item0 + qq;
      if (col < N) A[i + col * lda] = S[qq * ls + i];
    }
  }
  (void)valid;
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

lu_status launch_diag_crout(cudaStream_t st, float* a, int64_t lda, int w,
                            int64_t col0, int* first_bad) {
  if (w <= 0 || w > 128) return LU_ERR_INVALID_ARG;
  const int LD = ((w + 3) / 4) * 4 + 4;
  const size_t sm = ((size_t)LD * w + 8) * sizeof(float);
  LUB_CUDA_TRY(set_smem_limit((const void*)diag_crout_kernel, sm));
  diag_crout_kernel<<<1, kThreads, sm, st>>>(a, lda, w, col0, first_bad);
  LUB_LAUNCH_CHECK();
  return LU_SUCCESS;
}

static size_t lupanel_smem_bytes(int w) {
  const size_t wp = (size_t)((w + 7) / 8) * 8;
  return (wp * (wp + 4) + wp + (size_t)kItems * (wp + 4)) * sizeof(float);
}

lu_status launch_lupanel(cudaStream_t st, float* dg, int64_t lda, int w,
                         int64_t M, int64_t N, bool left) {
  if (w <= 0 || w > 128) return LU_ERR_INVALID_ARG;
  const int64_t nL = M > 0 ? ceil_div(M, kItems) : 0;
  const int64_t nU = N > 0 ? ceil_div(N, kItems) : 0;
  if (nL + nU == 0) return LU_SUCCESS;
  const size_t sm = lupanel_smem_bytes(w);
  LUB_CUDA_TRY(set_smem_limit((const void*)lupanel_kernel, sm));
  lupanel_kernel<<<(unsigned)(nL + nU), kPanelT, sm, st>>>(dg, lda, w, M, N, (int)nL,
                                                           left);
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
