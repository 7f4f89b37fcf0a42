// Inner (ib = 8) elimination of a block column held in shared memory, rows
// owned by threads: the reference's per-element order
// (src/lu_nopiv.cu:105-326, src/lu_nopiv_inner_rl.hxx:104-196) -- the 8x8
// diagonal tile (1/d correctly rounded, a multiply, fused a - l*u), the U
// columns right of it (forward substitution), the L rows below (row * 1/d
// and fused updates), then a rank-8 update accumulated acc = fma(l, u, acc)
// and subtracted once -- with one CTA barrier per 8 columns: the warp owning
// the next tile's rows factors it (one lane, in registers) while the other
// warps finish the current rank-8 update.  Used by the batched LU (block
// columns of up to 512 rows) and by the diagonal-block kernel of the single
// factorization.
#pragma once

#include "common.cuh"

namespace lub {
namespace rows {

__device__ __forceinline__ void load8(const float* p, float (&v)[8]) {
  const float4 a = *reinterpret_cast<const float4*>(p);
  const float4 b = *reinterpret_cast<const float4*>(p + 4);
  v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
  v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
}


// Owner warp of tile t: one lane factors the 8x8 tile in registers (no
// shuffles on the dependency chain), then the U strip (rows t0..t0+7,
// columns t0+8 .. wj-1, one column per lane).
__device__ __forceinline__ void tile_factor(float* C, int ldc, int c0, int t0,
                                            int wj, float* inv, int* bad, int pbase) {
  const int lane = threadIdx.x & 31;
  const int tw = min(8, wj - t0);
  float* T = C + (c0 + t0);
  if (lane == (t0 & 31) && !(tw == 8 && factor_tile8_fast(T + t0 * ldc, ldc, inv))) {
    // partial tile, or a pivot outside the fast range: the exact path
    float v[8][8];  // v[c][r]: tile column c
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      if (c < tw) {
        load8(T + (t0 + c) * ldc, v[c]);
      } else {
#pragma unroll
        for (int r = 0; r < 8; ++r) v[c][r] = 0.0f;
      }
    }
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      if (k < tw) {
        const float d = v[k][k];
        note_pivot(d, pbase + t0 + k, bad);
        const float iv = rcp_rn(d);  // correctly rounded 1/d
        inv[k] = iv;
#pragma unroll
        for (int r = k + 1; r < 8; ++r) v[k][r] = __fmul_rn(v[k][r], iv);
#pragma unroll
        for (int c = k + 1; c < 8; ++c)
#pragma unroll
          for (int r = k + 1; r < 8; ++r) v[c][r] = __fmaf_rn(-v[k][r], v[c][k], v[c][r]);
      }
    }
    // rows r >= tw of a partial tile lie below the matrix: never stored
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      if (c < tw) {
        if (tw == 8) {
          *reinterpret_cast<float4*>(T + (t0 + c) * ldc) =
              make_float4(v[c][0], v[c][1], v[c][2], v[c][3]);
          *reinterpret_cast<float4*>(T + (t0 + c) * ldc + 4) =
              make_float4(v[c][4], v[c][5], v[c][6], v[c][7]);
        } else {
#pragma unroll
          for (int r = 0; r < 8; ++r)
            if (r < tw) T[r + (t0 + c) * ldc] = v[c][r];
        }
      }
    }
  }
  __syncwarp();
  for (int c = t0 + 8 + lane; c < wj; c += 32) {
    float col[8];
    load8(T + c * ldc, col);
#pragma unroll
    for (int kk = 0; kk < 7; ++kk) {
      float l[8];
      load8(T + (t0 + kk) * ldc, l);  // tile column kk: l[r] = L[r][kk]
#pragma unroll
      for (int r = kk + 1; r < 8; ++r) col[r] = __fmaf_rn(-l[r], col[kk], col[r]);
    }
    *reinterpret_cast<float4*>(T + c * ldc) = make_float4(col[0], col[1], col[2], col[3]);
    *reinterpret_cast<float4*>(T + c * ldc + 4) = make_float4(col[4], col[5], col[6], col[7]);
  }
}

// Rows pa (and pb when TWO) below tile t (tw == 8): L elimination with the
// tile's U part and 1/d, then the rank-8 update of columns t0+8 .. wj-1.  Two
// rows share every shared-memory read of the tile and the U strip.
template <bool TWO>
__device__ __forceinline__ void row_update(float* C, int ldc, int c0, int t0, int wj,
                                           int pa, int pb, const float* inv) {
  float* ra_p = C + (c0 + pa);
  float* rb_p = C + (c0 + pb);
  const float* T = C + (c0 + t0);
  float ra[8], rb[8], iv[8];
  load8(inv, iv);
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    ra[c] = ra_p[(t0 + c) * ldc];
    rb[c] = TWO ? rb_p[(t0 + c) * ldc] : 0.0f;
  }
  // element c: fused updates with k = 0 .. c-1, then the 1/d multiply
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    float u[8];
    load8(T + (t0 + c) * ldc, u);  // u[k] = U[k][c]
#pragma unroll
    for (int k = 0; k < c; ++k) {
      ra[c] = __fmaf_rn(-ra[k], u[k], ra[c]);
      if (TWO) rb[c] = __fmaf_rn(-rb[k], u[k], rb[c]);
    }
    ra[c] = __fmul_rn(ra[c], iv[c]);
    if (TWO) rb[c] = __fmul_rn(rb[c], iv[c]);
  }
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    ra_p[(t0 + c) * ldc] = ra[c];
    if (TWO) rb_p[(t0 + c) * ldc] = rb[c];
  }
  int c = t0 + 8;
#pragma unroll 1
  for (; c + 4 <= wj; c += 4) {
    float u[4][8], acca[4], accb[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      load8(T + (c + j) * ldc, u[j]);
      acca[j] = 0.0f;
      accb[j] = 0.0f;
    }
#pragma unroll
    for (int k = 0; k < 8; ++k)
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        acca[j] = __fmaf_rn(ra[k], u[j][k], acca[j]);
        if (TWO) accb[j] = __fmaf_rn(rb[k], u[j][k], accb[j]);
      }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      ra_p[(c + j) * ldc] = __fsub_rn(ra_p[(c + j) * ldc], acca[j]);
      if (TWO) rb_p[(c + j) * ldc] = __fsub_rn(rb_p[(c + j) * ldc], accb[j]);
    }
  }
  for (; c < wj; ++c) {
    float u[8];
    load8(T + c * ldc, u);
    float acca = 0.0f, accb = 0.0f;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      acca = __fmaf_rn(ra[k], u[k], acca);
      if (TWO) accb = __fmaf_rn(rb[k], u[k], accb);
    }
    ra_p[c * ldc] = __fsub_rn(ra_p[c * ldc], acca);
    if (TWO) rb_p[c * ldc] = __fsub_rn(rb_p[c * ldc], accb);
  }
}

// Rows of the panel are dealt to the NT threads: row p < NT to thread p, and
// row NT + j to thread NT - 1 - j, so the warps that own the diagonal tiles
// (the first rows) take second rows last.  inv2: 2 x 8 floats (16-byte
// aligned) in shared memory; zero / non-finite pivots are reported to *bad
// as 1-based column pbase + k.
template <int NT>
__device__ __forceinline__ void panel_block(float* C, int ldc, int n, int c0, int wj,
                                            float* inv2, int* bad, int pbase) {
  constexpr int kWarpsP = NT / 32;
  const int tid = threadIdx.x, warp = tid >> 5;
  const int M = n - c0;
  const int nt = (wj + 7) >> 3;
  const int pa = tid, pb = NT + (NT - 1 - tid);
  if (warp == 0) tile_factor(C, ldc, c0, 0, wj, inv2, bad, pbase);
  __syncthreads();
#pragma unroll 1
  for (int t = 0; t < nt; ++t) {
    const int t0 = 8 * t;
    const float* inv = inv2 + 8 * (t & 1);
    // rows exist below tile t only when it is a full tile
    const bool ha = pa >= t0 + 8 && pa < M;
    const bool hb = pb < M;  // pb >= NT > t0 + 8
    const bool lookahead = t + 1 < nt && warp == (((t0 + 8) >> 5) % kWarpsP);
    if (lookahead) {
      // this warp owns tile t+1: update its first rows (which include the
      // tile's) and factor the tile while the other warps finish chunk t
      if (ha) row_update<false>(C, ldc, c0, t0, wj, pa, pa, inv);
      tile_factor(C, ldc, c0, t0 + 8, wj, inv2 + 8 * ((t + 1) & 1), bad, pbase);
      if (hb) row_update<false>(C, ldc, c0, t0, wj, pb, pb, inv);
    } else if (ha && hb) {
      row_update<true>(C, ldc, c0, t0, wj, pa, pb, inv);
    } else if (ha || hb) {
      const int p = ha ? pa : pb;
      row_update<false>(C, ldc, c0, t0, wj, p, p, inv);
    }
    __syncthreads();
  }
}

}  // namespace rows
}  // namespace lub
