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
//   diag_factor_kernel : the w x w diagonal block, one CTA, in shared memory
//                        (diag_crout_kernel: the same for the left-looking
//                        variant's Crout order);
//   lupanel_kernel     : the L21 rows below the block and the U12 columns
//                        right of it, 64 rows or 64 columns per CTA (one grid
//                        for both strips), optionally writing the K-major
//                        tensor-core operand copies of what it finishes;
//   ref_panel_kernel   : remifa::lu_nopiv_panel<float,8> as a standalone
//                        entry point (lu_panel_c);
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
// diag_factor_kernel: threads 0-255 eliminate the L rows / U columns of a
// tile, threads 32-511 its trailing rank-8 update (16 warps hide the shared
// memory latency of the 4 x 4 micro-tiles).
constexpr int kDiagT = 512;

// Block copies between global memory and shared memory, by all NT threads
// of the CTA: warps take columns, lanes consecutive rows, so no index is
// divided by a runtime extent.  Both sides column-major unless noted.

// dst[r + c*ldd] = src[r + c*lds] asynchronously (complete with
// cp_async_wait_all); 16-byte copies when every column start is 16-byte
// aligned on both sides.
template <int NT>
__device__ __forceinline__ void stage_cols_async(float* dst, int ldd, const float* src,
                                                 int64_t lds, int rows, int cols) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int kNW = NT / 32;
  const bool vec = ((reinterpret_cast<uintptr_t>(src) | reinterpret_cast<uintptr_t>(dst)) & 15) == 0 &&
                   (lds & 3) == 0 && (ldd & 3) == 0 && (rows & 3) == 0;
  if (vec) {
    for (int c = warp; c < cols; c += kNW) {
      const float* s = src + (int64_t)c * lds;
      float* d = dst + c * ldd;
      for (int r = 4 * lane; r < rows; r += 128) cp_async16(d + r, s + r);
    }
  } else {
    for (int c = warp; c < cols; c += kNW) {
      const float* s = src + (int64_t)c * lds;
      float* d = dst + c * ldd;
      for (int r = lane; r < rows; r += 32) cp_async4(d + r, s + r);
    }
  }
}

// dst[r + c*ldd] = src[r + c*lds] (shared -> global), 16-byte stores when
// every column start is 16-byte aligned on both sides.
template <int NT>
__device__ __forceinline__ void store_cols(float* dst, int64_t ldd, const float* src,
                                           int lds, int rows, int cols) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int kNW = NT / 32;
  const bool vec = ((reinterpret_cast<uintptr_t>(src) | reinterpret_cast<uintptr_t>(dst)) & 15) == 0 &&
                   (ldd & 3) == 0 && (lds & 3) == 0 && (rows & 3) == 0;
  if (vec) {
    for (int c = warp; c < cols; c += kNW) {
      const float* s = src + c * lds;
      float* d = dst + (int64_t)c * ldd;
      for (int r = 4 * lane; r < rows; r += 128)
        *reinterpret_cast<float4*>(d + r) = *reinterpret_cast<const float4*>(s + r);
    }
  } else {
    for (int c = warp; c < cols; c += kNW) {
      const float* s = src + c * lds;
      float* d = dst + (int64_t)c * ldd;
      for (int r = lane; r < rows; r += 32) d[r] = s[r];
    }
  }
}

// Transposing load: dst[r*ldd + c] = src[r + c*lds] for r < rows, c < cols,
// and 0 for cols <= c < round4(cols).  Each thread reads four columns of
// one row (coalesced across the lanes) and writes them as one 16-byte
// shared store; dst 16-byte aligned, ldd % 4 == 0.
template <int NT>
__device__ __forceinline__ void stage_rows_t(float* dst, int ldd, const float* src,
                                             int64_t lds, int rows, int cols) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int kNW = NT / 32;
  const int nq = (cols + 3) >> 2;
  for (int q = warp; q < nq; q += kNW) {
    const int c0 = 4 * q;
    const float* s = src + (int64_t)c0 * lds;
#pragma unroll 2
    for (int r = lane; r < rows; r += 32) {
      float v[4];
#pragma unroll
      for (int e = 0; e < 4; ++e) v[e] = (c0 + e < cols) ? s[r + e * lds] : 0.0f;
      *reinterpret_cast<float4*>(dst + r * ldd + c0) = make_float4(v[0], v[1], v[2], v[3]);
    }
  }
}

// Transposing store: dst[r + c*ldd] = src[r*lds + c] for r < rows,
// c < cols (16-byte shared reads; src 16-byte aligned, lds % 4 == 0).
template <int NT>
__device__ __forceinline__ void store_rows_t(float* dst, int64_t ldd, const float* src,
                                             int lds, int rows, int cols) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int kNW = NT / 32;
  const int nq = (cols + 3) >> 2;
  for (int q = warp; q < nq; q += kNW) {
    const int c0 = 4 * q;
    float* d = dst + (int64_t)c0 * ldd;
#pragma unroll 2
    for (int r = lane; r < rows; r += 32) {
      const float4 v4 = *reinterpret_cast<const float4*>(src + r * lds + c0);
      const float v[4] = {v4.x, v4.y, v4.z, v4.w};
#pragma unroll
      for (int e = 0; e < 4; ++e)
        if (c0 + e < cols) d[r + e * ldd] = v[e];
    }
  }
}

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
      const float iv = rcp_rn(d);  // correctly rounded 1/d
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
      const float iv = rcp_rn(d);  // correctly rounded 1/d
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
__global__ void __launch_bounds__(kDiagT)
diag_factor_kernel(float* __restrict__ a, int64_t lda, int w, int64_t col0,
                   int* first_bad) {
  extern __shared__ __align__(16) float smem[];
  const int LD = ((w + 3) / 4) * 4 + 4;
  float* D = smem;
  float* Ls = D + (size_t)LD * w;     // [8][128]
  float* Us = Ls + 8 * 128;           // [8][128]
  float* inv = Us + 8 * 128;          // [8]
  const int tid = threadIdx.x;

  stage_cols_async<kDiagT>(D, LD, a, lda, w, w);
  cp_async_wait_all();
  __syncthreads();

  const int nt = (w + 7) / 8;
  // Phase A of tile 0: one thread factors the 8 x 8 tile in registers
  // (src/lu_nopiv.cu:123-171): 1/d, scale the column below, fused rank-1
  // update of the rest of the tile.  Later tiles are factored during the
  // previous tile's Phase C (look-ahead, below).
  if (tid == 0) {
    const int tw0 = min(8, w);
    if (!(tw0 == 8 && factor_tile8_fast(D, LD, inv)))
      factor_tile_thread(D, LD, tw0, inv, col0, first_bad);
  }
  __syncthreads();
  for (int t = 0; t < nt; ++t) {
    const int t0 = 8 * t;
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
    // Look-ahead: warp 0 updates the next tile's 8 x 8 block (two elements
    // per lane) and its lane 0 factors it, while warps 1.. update the rest.
    const int t1w = min(8, s);  // width of tile t+1
    if (tid < 32) {
      float* T1 = D + (t0 + 8) + (t0 + 8) * LD;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int e = tid + 32 * h, i = e & 7, j = e >> 3;
        if (i < t1w && j < t1w) {
          float acc = 0.0f;
#pragma unroll
          for (int k = 0; k < 8; ++k) acc = __fmaf_rn(Ls[k * 128 + i], Us[k * 128 + j], acc);
          T1[i + j * LD] = __fsub_rn(T1[i + j * LD], acc);
        }
      }
      __syncwarp();
      if (tid == 0 && !(t1w == 8 && factor_tile8_fast(T1, LD, inv)))
        factor_tile_thread(T1, LD, t1w, inv, col0 + t0 + 8, first_bad);
    }
    const int nb4 = (s + 3) / 4;
    const bool vec = (s % 4 == 0);
    for (int b = tid - 32; b < nb4 * nb4; b += kDiagT - 32) {
      if (b < 0) break;
      const int li = 4 * (b % nb4), lj = 4 * (b / nb4);  // local to the block
      if (li < 8 && lj < 8) continue;  // the next tile: thread 0
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

  store_cols<kDiagT>(a, lda, D, LD, w, w);
}

// ---------------------------------------------------------------------------
// Diagonal block of the left-looking (Crout) variant, w <= 128, one CTA.
// The reference's order (src/lu_nopiv_inner_ll.hxx:197-370), per tile T:
// the tile column (rows >= 8T) and the tile row (columns right of the tile)
// receive one update summing all earlier columns of the block (acc =
// sum_k fma(L[i][k], U[k][j], acc) from 0 over k < 8T, subtracted once),
// then the tile is factored and the L rows / U columns of the block are
// eliminated with it.  Each element's sum is one fma chain in k order, so
// it can be carried along tile by tile: ACC (w x w) holds every trailing
// element's chain, extended by each tile's 8 columns as soon as the tile's
// L rows / U columns are known (a rank-8 step over the whole trailing block,
// like diag_factor_kernel's Phase C, with ACC in place of the subtraction)
// and subtracted from the element when its own tile comes.  Bit for bit the
// reference's sums and subtractions; the work per tile is spread over the
// whole trailing block instead of the tile's column and row.
__global__ void __launch_bounds__(kDiagT)
diag_crout_kernel(float* __restrict__ a, int64_t lda, int w, int64_t col0,
                  int* first_bad) {
  extern __shared__ __align__(16) float smem[];
  const int LD = ((w + 3) / 4) * 4 + 4;
  float* D = smem;
  float* ACC = D + (size_t)LD * w;
  float* Ls = ACC + (size_t)LD * w;   // [8][128]
  float* Us = Ls + 8 * 128;           // [8][128]
  float* inv = Us + 8 * 128;          // [8]
  const int tid = threadIdx.x;

  stage_cols_async<kDiagT>(D, LD, a, lda, w, w);
  for (int i = tid; i < LD * w; i += kDiagT) ACC[i] = 0.0f;
  cp_async_wait_all();
  __syncthreads();

  // tile 0: no earlier columns
  if (tid == 0) {
    const int tw0 = min(8, w);
    if (!(tw0 == 8 && factor_tile8_fast(D, LD, inv)))
      factor_tile_thread(D, LD, tw0, inv, col0, first_bad);
  }
  __syncthreads();
  const int nt = (w + 7) / 8;
  for (int t = 0; t < nt; ++t) {
    const int t0 = 8 * t;
    const int s = w - t0 - 8;  // trailing extent inside the block
    if (s <= 0) break;
    // The tile's L rows below it (threads 0..127) and U columns right of it
    // (threads 128..255): first the subtraction of the element's sum over
    // the earlier tiles, then the elimination with the tile; results also
    // go to the strip buffers.
    if (tid < 128) {
      if (tid < s) {
        const int i = t0 + 8 + tid;
        float row[8];
#pragma unroll
        for (int c = 0; c < 8; ++c) {
          row[c] = D[i + (t0 + c) * LD];
          if (t0 > 0) row[c] = __fsub_rn(row[c], ACC[i + (t0 + c) * LD]);
        }
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          row[k] = __fmul_rn(row[k], inv[k]);
#pragma unroll
          for (int c = k + 1; c < 8; ++c)
            row[c] = __fmaf_rn(-row[k], D[(t0 + k) + (t0 + c) * LD], row[c]);
        }
#pragma unroll
        for (int c = 0; c < 8; ++c) {
          D[i + (t0 + c) * LD] = row[c];
          Ls[c * 128 + (i - t0 - 8)] = row[c];
        }
      }
    } else if (tid < 256) {
      const int q = tid - 128;
      if (q < s) {
        const int j = t0 + 8 + q;
        float col[8];
#pragma unroll
        for (int r = 0; r < 8; ++r) {
          col[r] = D[(t0 + r) + j * LD];
          if (t0 > 0) col[r] = __fsub_rn(col[r], ACC[(t0 + r) + j * LD]);
        }
#pragma unroll
        for (int k = 0; k < 8; ++k)
#pragma unroll
          for (int r = k + 1; r < 8; ++r)
            col[r] = __fmaf_rn(-D[(t0 + r) + (t0 + k) * LD], col[k], col[r]);
#pragma unroll
        for (int r = 0; r < 8; ++r) {
          D[(t0 + r) + j * LD] = col[r];
          Us[r * 128 + q] = col[r];
        }
      }
    }
    __syncthreads();
    // The tile's 8 columns appended to every trailing element's sum.
    // Look-ahead: warp 0 finishes the next tile's block (its sum, one
    // subtraction) and its lane 0 factors it, while warps 1.. extend ACC.
    const int t1w = min(8, s);  // width of tile t+1
    if (tid < 32) {
      float* T1 = D + (t0 + 8) + (t0 + 8) * LD;
      const float* A1 = ACC + (t0 + 8) + (t0 + 8) * LD;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int e = tid + 32 * h, i = e & 7, j = e >> 3;
        if (i < t1w && j < t1w) {
          float acc = A1[i + j * LD];
#pragma unroll
          for (int k = 0; k < 8; ++k) acc = __fmaf_rn(Ls[k * 128 + i], Us[k * 128 + j], acc);
          T1[i + j * LD] = __fsub_rn(T1[i + j * LD], acc);
        }
      }
      __syncwarp();
      if (tid == 0 && !(t1w == 8 && factor_tile8_fast(T1, LD, inv)))
        factor_tile_thread(T1, LD, t1w, inv, col0 + t0 + 8, first_bad);
    }
    const int nb4 = (s + 3) / 4;
    const bool vec = (s % 4 == 0);
    for (int b = tid - 32; b < nb4 * nb4; b += kDiagT - 32) {
      if (b < 0) break;
      const int li = 4 * (b % nb4), lj = 4 * (b / nb4);  // local to the block
      if (li < 8 && lj < 8) continue;  // the next tile: warp 0
      const int i0 = t0 + 8 + li, j0 = t0 + 8 + lj;
      float acc[4][4];
      if (vec) {
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) {
          const float4 c4 = *reinterpret_cast<const float4*>(&ACC[i0 + (j0 + jj) * LD]);
          acc[0][jj] = c4.x; acc[1][jj] = c4.y; acc[2][jj] = c4.z; acc[3][jj] = c4.w;
        }
      } else {
#pragma unroll
        for (int ii = 0; ii < 4; ++ii)
#pragma unroll
          for (int jj = 0; jj < 4; ++jj)
            acc[ii][jj] = (i0 + ii < w && j0 + jj < w) ? ACC[(i0 + ii) + (j0 + jj) * LD] : 0.0f;
      }
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const float4 l4 = *reinterpret_cast<const float4*>(&Ls[k * 128 + li]);
        const float4 u4 = *reinterpret_cast<const float4*>(&Us[k * 128 + lj]);
        const float l[4] = {l4.x, l4.y, l4.z, l4.w};
        const float u[4] = {u4.x, u4.y, u4.z, u4.w};
#pragma unroll
        for (int ii = 0; ii < 4; ++ii)
#pragma unroll
          for (int jj = 0; jj < 4; ++jj) acc[ii][jj] = __fmaf_rn(l[ii], u[jj], acc[ii][jj]);
      }
      if (vec) {
#pragma unroll
        for (int jj = 0; jj < 4; ++jj)
          *reinterpret_cast<float4*>(&ACC[i0 + (j0 + jj) * LD]) =
              make_float4(acc[0][jj], acc[1][jj], acc[2][jj], acc[3][jj]);
      } else {
#pragma unroll
        for (int ii = 0; ii < 4; ++ii)
#pragma unroll
          for (int jj = 0; jj < 4; ++jj)
            if (i0 + ii < w && j0 + jj < w) ACC[(i0 + ii) + (j0 + jj) * LD] = acc[ii][jj];
      }
    }
    __syncthreads();
  }

  store_cols<kDiagT>(a, lda, D, LD, w, w);
}

// ---------------------------------------------------------------------------
// L and U panels of one sub-panel, one launch.  `dg` is the factored w x w
// diagonal block (lda); M rows lie below it (L21), N columns right of it
// (U12).  A CTA owns kItems rows of L21 or columns of U12 ("items"), each
// item's w values held contiguously in shared memory (S[item][pos]), and
// walks the 8-wide tiles T left to right:
//   (a) one thread per item eliminates tile T of its item: L rows
//       x_k *= 1/d_k, x_j -= x_k U[k][j] (src/lu_nopiv.cu:141-168); U
//       columns x_j -= L[j][k] x_k (src/lu_nopiv.cu:304-316);
//   (b) the rank-8 update of tile T to the item positions right of it,
//       acc = sum_k fma(x_k, F_k) over the tile's 8 columns then one
//       subtraction -- the reference's K = 8 GEMMs; the positions of tile
//       T+1 are updated and eliminated first, by the item threads, while
//       the other warps update the rest (lupanel_strip).
// Each element receives the reference's operations in the reference's
// order.  Left-looking mode (src/lu_nopiv_inner_ll.hxx:225-300) keeps one
// running sum per element across the earlier tiles (ACC) and subtracts it
// once, just before the element's tile is eliminated.
constexpr int kPanelT = 256;
constexpr int kItems = 64;                 // rows / columns per CTA
constexpr int kMicroI = 4, kMicroP = 8;    // register micro-tile

__device__ __forceinline__ void ld8(const float* p, float (&v)[8]) {
  const float4 a = *reinterpret_cast<const float4*>(p);
  const float4 b = *reinterpret_cast<const float4*>(p + 4);
  v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
  v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
}
__device__ __forceinline__ void st8(float* p, const float (&v)[8]) {
  *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
  *reinterpret_cast<float4*>(p + 4) = make_float4(v[4], v[5], v[6], v[7]);
}

// Eliminate tile columns [t0, t0 + tw) of one item held in x[0..8):
// L rows x_c -= x_k U[k][c] (k < c), then x_c *= 1/d_c
// (src/lu_nopiv.cu:141-168); U columns x_c -= L[c][k] x_k
// (src/lu_nopiv.cu:304-316).
template <bool IS_L>
__device__ __forceinline__ void lupanel_elim(const float* F, int lf, const float* inv,
                                             int t0, int tw, float (&x)[8]) {
  if (tw == 8) {
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      float f[8];
      ld8(F + (t0 + c) * lf + t0, f);  // f[k] = U[k][c] (L) / L[c][k] (U)
      if (IS_L) {
#pragma unroll
        for (int k = 0; k < c; ++k) x[c] = __fmaf_rn(-x[k], f[k], x[c]);
        x[c] = __fmul_rn(x[c], inv[t0 + c]);
      } else {
#pragma unroll
        for (int k = 0; k < c; ++k) x[c] = __fmaf_rn(-f[k], x[k], x[c]);
      }
    }
  } else {
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      if (c < tw) {
        const float* f = F + (t0 + c) * lf + t0;
        if (IS_L) {
#pragma unroll
          for (int k = 0; k < c; ++k) x[c] = __fmaf_rn(-x[k], f[k], x[c]);
          x[c] = __fmul_rn(x[c], inv[t0 + c]);
        } else {
#pragma unroll
          for (int k = 0; k < c; ++k) x[c] = __fmaf_rn(-f[k], x[k], x[c]);
        }
      }
    }
  }
}

// F[pos * lf + k]: the factor values that multiply item value k for
// position pos -- U[k][pos] (L blocks, F column-major) or L[pos][k] (U
// blocks, F row-major) -- so the 8 values of one tile are two float4.
// Per tile T, after one barrier:
//   warps 0-1 (one thread per item) apply tile T's rank-8 update to the
//     8 positions of tile T+1 and eliminate tile T+1 at once (look-ahead);
//   warps 2-7 apply tile T's rank-8 update to the positions right of tile
//     T+1 in register micro-tiles of 4 items x 8 positions (256 FMAs per 24
//     vector loads).
// Every element still receives acc = sum_k fma(x_k, F_k) over the tile's 8
// columns in k order, then one subtraction (left-looking: one running sum,
// subtracted just before the element's own tile is eliminated).
template <bool IS_L, bool LEFT>
__device__ __forceinline__ void lupanel_strip(const float* F, int lf, const float* inv,
                                              float* S, int ls, float* ACC, int w) {
  constexpr int kIG = kItems / kMicroI;  // 16 item groups
  const int tid = threadIdx.x;
  const int nt = (w + 7) / 8;
  if (tid < kItems) {  // tile 0
    float* xr = S + tid * ls;
    float x[8];
    ld8(xr, x);
    lupanel_elim<IS_L>(F, lf, inv, 0, min(8, w), x);
    st8(xr, x);
  }
  __syncthreads();
  for (int T = 0; T + 1 < nt; ++T) {
    const int t0 = 8 * T, p0 = t0 + 8;
    if (tid < kItems) {
      float* xr = S + tid * ls;
      float xv[8], x[8], acc[8];
      ld8(xr + t0, xv);
      ld8(xr + p0, x);
      if (LEFT) {
        ld8(ACC + tid * ls + p0, acc);
      } else {
#pragma unroll
        for (int b = 0; b < 8; ++b) acc[b] = 0.0f;
      }
#pragma unroll
      for (int b = 0; b < 8; ++b) {
        float f[8];
        ld8(F + (p0 + b) * lf + t0, f);
#pragma unroll
        for (int k = 0; k < 8; ++k) acc[b] = __fmaf_rn(xv[k], f[k], acc[b]);
      }
#pragma unroll
      for (int b = 0; b < 8; ++b) x[b] = __fsub_rn(x[b], acc[b]);
      lupanel_elim<IS_L>(F, lf, inv, p0, min(8, w - p0), x);
      st8(xr + p0, x);
    } else {
      const int q0 = p0 + 8;
      const int npos = (w - q0 + kMicroP - 1) / kMicroP;
      for (int m = tid - kItems; m < npos * kIG; m += kPanelT - kItems) {
        const int ig = m % kIG, pp = q0 + (m / kIG) * kMicroP;
        float xv[kMicroI][8];
#pragma unroll
        for (int a = 0; a < kMicroI; ++a) ld8(S + (ig + a * kIG) * ls + t0, xv[a]);
        float acc[kMicroI][kMicroP];
#pragma unroll
        for (int a = 0; a < kMicroI; ++a) {
          if (LEFT) {
            ld8(ACC + (ig + a * kIG) * ls + pp, acc[a]);
          } else {
#pragma unroll
            for (int b = 0; b < kMicroP; ++b) acc[a][b] = 0.0f;
          }
        }
#pragma unroll
        for (int b = 0; b < kMicroP; ++b) {
          float f[8];
          ld8(F + (pp + b) * lf + t0, f);
#pragma unroll
          for (int k = 0; k < 8; ++k)
#pragma unroll
            for (int a = 0; a < kMicroI; ++a) acc[a][b] = __fmaf_rn(xv[a][k], f[k], acc[a][b]);
        }
#pragma unroll
        for (int a = 0; a < kMicroI; ++a) {
          float* row = (LEFT ? ACC : S) + (ig + a * kIG) * ls + pp;
          if (LEFT) {
            st8(row, acc[a]);
          } else {
            float c[8];
            ld8(row, c);
#pragma unroll
            for (int b = 0; b < kMicroP; ++b) c[b] = __fsub_rn(c[b], acc[a][b]);
            st8(row, c);
          }
        }
      }
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kPanelT)
lupanel_kernel(float* __restrict__ dg, int64_t lda, int w, int64_t M,
               int64_t N, int nL, bool left, int64_t offL, int64_t offU, LuPack pk) {
  extern __shared__ __align__(16) float smem[];
  const int tid = threadIdx.x;
  const int wp = ((w + 7) / 8) * 8;  // padded width (zero filled)
  const int ls = wp + 4;             // item stride (breaks bank aliasing)
  const int lf = wp + 4;             // leading dimension of F, same reason
  float* F = smem;                   // diagonal block, wp x wp
  float* inv = F + (size_t)wp * lf;  // wp
  float* S = inv + wp;               // kItems x ls
  float* ACC = S + (size_t)kItems * ls;  // left-looking running sums
  const bool is_l = (int)blockIdx.x < nL;

  // Stage the factored diagonal block: column-major (F[c*lf + r]) for L
  // blocks, row-major (F[r*lf + c]) for U blocks; the padding rows and
  // columns [w, wp) are zero.
  if (is_l) stage_cols_async<kPanelT>(F, lf, dg, lda, w, w);
  else stage_rows_t<kPanelT>(F, lf, dg, lda, w, w);
  if (wp != w) {
    for (int idx = tid; idx < wp * wp; idx += kPanelT) {
      const int r = idx % wp, c = idx / wp;
      if (r >= w || c >= (is_l ? w : ((w + 3) & ~3))) F[is_l ? c * lf + r : r * lf + c] = 0.0f;
    }
  }
  int64_t item0;
  float* A;
  int nitems;
  if (is_l) {
    item0 = (int64_t)blockIdx.x * kItems;
    A = dg + w + offL;               // first row of this launch's L rows
    nitems = (int)std::min<int64_t>(kItems, M - item0);
    // S[q*ls + c] = A[row item0 + q, column c]
    stage_rows_t<kPanelT>(S, ls, A + item0, lda, nitems, w);
  } else {
    item0 = (int64_t)(blockIdx.x - nL) * kItems;
    A = dg + (w + offU) * lda;       // first column of this launch's U columns
    nitems = (int)std::min<int64_t>(kItems, N - item0);
    // S[q*ls + i] = A[row i, column item0 + q]
    stage_cols_async<kPanelT>(S, ls, A + item0 * lda, lda, w, nitems);
  }
  // zero the positions [w, wp) of every item and the items past the end
  {
    const int wq = is_l ? ((w + 3) & ~3) : w;  // the L staging zeroed up to round4(w)
    const int padc = wp - wq;
    if (padc > 0)
      for (int idx = tid; idx < kItems * padc; idx += kPanelT)
        S[(idx / padc) * ls + wq + idx % padc] = 0.0f;
    for (int idx = nitems * ls + tid; idx < kItems * ls; idx += kPanelT) S[idx] = 0.0f;
  }
  if (left)
    for (int idx = tid; idx < kItems * ls; idx += kPanelT) ACC[idx] = 0.0f;
  cp_async_wait_all();
  __syncthreads();
  if (is_l) {
    for (int k = tid; k < wp; k += kPanelT)
      inv[k] = (k < w) ? rcp_rn(F[k * lf + k]) : 0.0f;
    __syncthreads();
    if (left) lupanel_strip<true, true>(F, lf, inv, S, ls, ACC, w);
    else lupanel_strip<true, false>(F, lf, inv, S, ls, ACC, w);
  } else {
    if (left) lupanel_strip<false, true>(F, lf, inv, S, ls, ACC, w);
    else lupanel_strip<false, false>(F, lf, inv, S, ls, ACC, w);
  }
  if (is_l) store_rows_t<kPanelT>(A + item0, lda, S, ls, nitems, w);
  else store_cols<kPanelT>(A + item0 * lda, lda, S, ls, w, nitems);
  // the finished items as tensor-core operands: item qq's w values are
  // contiguous along K in both copies (consecutive threads, consecutive k)
  // destination 0: the tensor-core operand copy; 1: the second L copy
  for (int dsel = 0; dsel < 2; ++dsel) {
    void* dst = dsel == 0 ? (is_l ? pk.pa : pk.pb) : (is_l ? pk.pa2 : nullptr);
    if (!dst) continue;
    const int64_t lim = is_l ? M : N;
    const int64_t base = (dsel == 1 ? pk.row02 : is_l ? pk.row0 : pk.col0) + item0;
    const int64_t ldk = dsel == 1 ? pk.ldk2 : pk.ldk;
    const int k0 = dsel == 1 ? pk.k02 : pk.k0;
    if (w % 8 == 0 && ldk % 8 == 0 && k0 % 8 == 0) {
      // 8 values -> one 16-byte store
      const int w8 = w / 8;  // <= 16
      for (int idx = tid; idx < kItems * 16; idx += kPanelT) {
        const int c8 = idx & 15, qq = idx >> 4;
        const int64_t pr = base + qq;
        if (c8 < w8 && item0 + qq < lim && pr >= 0) {
          float v[8];
          ld8(&S[qq * ls + 8 * c8], v);
          uint4 out;
          uint32_t* o32 = reinterpret_cast<uint32_t*>(&out);
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            if (pk.bf16) {
              const __nv_bfloat162 h = __floats2bfloat162_rn(v[2 * e], v[2 * e + 1]);
              o32[e] = *reinterpret_cast<const uint32_t*>(&h);
            } else {
              const __half2 h = __floats2half2_rn(v[2 * e], v[2 * e + 1]);
              o32[e] = *reinterpret_cast<const uint32_t*>(&h);
            }
          }
          *reinterpret_cast<uint4*>(static_cast<uint16_t*>(dst) + pr * ldk + k0 + 8 * c8) = out;
        }
      }
    } else {
      for (int idx = tid; idx < kItems * w; idx += kPanelT) {
        const int c = idx % w, qq = idx / w;
        const int64_t pr = base + qq;
        if (item0 + qq < lim && pr >= 0) {
          const float v = S[qq * ls + c];
          const int64_t o = pr * ldk + k0 + c;
          if (pk.bf16) static_cast<__nv_bfloat16*>(dst)[o] = __float2bfloat16_rn(v);
          else static_cast<__half*>(dst)[o] = __float2half_rn(v);
        }
      }
    }
  }
  (void)nitems;
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

// ---------------------------------------------------------------------------
// remifa::lu_nopiv_panel<half,8>: the same panel with fp16 storage and the
// reference's fp16 arithmetic (src/lu_nopiv.cu:105-326 instantiated for
// half, where nvcc contracts each a -= l * u into one fp16 fused multiply-add,
// which the reference's own outputs show): the pivot's reciprocal 1/d and
// the scaling l * (1/d) each rounded to fp16, and the update a - l * u
// rounded once.  The fp16 intrinsics below are the operations those
// expressions compile to.
__device__ __forceinline__ float h16_div1(float d) {
  return __half2float(__hdiv(__float2half(1.0f), __float2half(d)));
}
__device__ __forceinline__ float h16_mul(float a, float b) {
  return __half2float(__hmul(__float2half(a), __float2half(b)));
}
__device__ __forceinline__ float h16_sub_mul(float a, float l, float u) {
  return __half2float(__hfma(__hneg(__float2half(l)), __float2half(u), __float2half(a)));
}

__global__ void __launch_bounds__(kThreads)
ref_panel_f16_kernel(int64_t m, int n, const __half* __restrict__ d, int64_t ldd,
                     __half* __restrict__ l, int64_t ldl, __half* __restrict__ u,
                     int64_t ldu, int* stat) {
  __shared__ float T[8][9];
  __shared__ float inv[8];
  const int tid = threadIdx.x;
  if (tid < 64) {
    const int r = tid % 8, c = tid / 8;
    T[r][c] = (r < n && c < n) ? __half2float(d[r + c * ldd]) : 0.0f;
  }
  __syncthreads();
  if (tid == 0) {  // the 8 x 8 tile, right-looking, one thread (64 operations)
    for (int k = 0; k < n; ++k) {
      inv[k] = h16_div1(T[k][k]);
      for (int r = k + 1; r < n; ++r) T[r][k] = h16_mul(T[r][k], inv[k]);
      for (int c = k + 1; c < n; ++c)
        for (int r = k + 1; r < n; ++r) T[r][c] = h16_sub_mul(T[r][c], T[r][k], T[k][c]);
    }
  }
  __syncthreads();
  if (blockIdx.x == 0 && blockIdx.y == 0) {
    if (tid < 64) {
      const int r = tid % 8, c = tid / 8;
      if (r < n && c < n) l[r + c * ldl] = __float2half_rn(T[r][c]);
    }
    if (tid == 0 && stat) *stat = n;
  }
  const int64_t q = (int64_t)blockIdx.x * kThreads + tid + n;
  if (q >= m) return;
  if (blockIdx.y == 0) {
    float row[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) row[c] = (c < n) ? __half2float(l[q + c * ldl]) : 0.0f;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      if (k < n) {
        row[k] = h16_mul(row[k], inv[k]);
#pragma unroll
        for (int c = k + 1; c < 8; ++c)
          if (c < n) row[c] = h16_sub_mul(row[c], row[k], T[k][c]);
      }
    }
#pragma unroll
    for (int c = 0; c < 8; ++c)
      if (c < n) l[q + c * ldl] = __float2half_rn(row[c]);
  } else {
    float col[8];
#pragma unroll
    for (int r = 0; r < 8; ++r) col[r] = (r < n) ? __half2float(u[r + q * ldu]) : 0.0f;
#pragma unroll
    for (int k = 0; k < 8; ++k)
#pragma unroll
      for (int r = k + 1; r < 8; ++r)
        if (k < n && r < n) col[r] = h16_sub_mul(col[r], T[r][k], col[k]);
#pragma unroll
    for (int r = 0; r < 8; ++r)
      if (r < n) u[r + q * ldu] = __float2half_rn(col[r]);
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
  diag_factor_kernel<<<1, kDiagT, sm, st>>>(a, lda, w, col0, first_bad);
  LUB_LAUNCH_CHECK();
  return LU_SUCCESS;
}

lu_status launch_diag_crout(cudaStream_t st, float* a, int64_t lda, int w,
                            int64_t col0, int* first_bad) {
  if (w <= 0 || w > 128) return LU_ERR_INVALID_ARG;
  const int LD = ((w + 3) / 4) * 4 + 4;
  const size_t sm = ((size_t)2 * LD * w + 2 * 8 * 128 + 8) * sizeof(float);
  LUB_CUDA_TRY(set_smem_limit((const void*)diag_crout_kernel, sm));
  diag_crout_kernel<<<1, kDiagT, sm, st>>>(a, lda, w, col0, first_bad);
  LUB_LAUNCH_CHECK();
  return LU_SUCCESS;
}

static size_t lupanel_smem_bytes(int w, bool left) {
  const size_t wp = (size_t)((w + 7) / 8) * 8;
  return (wp * (wp + 4) + wp + (size_t)(left ? 2 : 1) * kItems * (wp + 4)) * sizeof(float);
}

lu_status launch_lupanel(cudaStream_t st, float* dg, int64_t lda, int w,
                         int64_t M, int64_t N, bool left, int64_t offL, int64_t offU,
                         const LuPack* pack) {
  if (w <= 0 || w > 128) return LU_ERR_INVALID_ARG;
  const int64_t nL = M > 0 ? ceil_div(M, kItems) : 0;
  const int64_t nU = N > 0 ? ceil_div(N, kItems) : 0;
  if (nL + nU == 0) return LU_SUCCESS;
  const size_t sm = lupanel_smem_bytes(w, left);
  LUB_CUDA_TRY(set_smem_limit((const void*)lupanel_kernel, sm));
  const LuPack pk = pack ? *pack : LuPack{};
  lupanel_kernel<<<(unsigned)(nL + nU), kPanelT, sm, st>>>(dg, lda, w, M, N, (int)nL,
                                                           left, offL, offU, pk);
  LUB_LAUNCH_CHECK();
  return LU_SUCCESS;
}

lu_status launch_ref_panel_f16(cudaStream_t st, int64_t m, int n, const __half* d,
                               int64_t ldd, __half* l, int64_t ldl, __half* u,
                               int64_t ldu, int* stat) {
  if (n <= 0 || n > 8 || m < n) return LU_ERR_INVALID_ARG;
  const int64_t rest = m - n;
  dim3 grid((unsigned)std::max<int64_t>(1, ceil_div(rest, kThreads)), 2);
  ref_panel_f16_kernel<<<grid, kThreads, 0, st>>>(m, n, d, ldd, l, ldl, u, ldu, stat);
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
