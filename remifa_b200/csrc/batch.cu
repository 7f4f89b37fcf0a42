// Batched no-pivot LU of many independent matrices of uneven size (new; the
// reference factors one matrix per call).
//
// One persistent launch: every CTA takes the next matrix from a work list
// (sorted by decreasing size so the large ones start first) through a
// global atomic counter, factors it alone, and takes the next.  Per matrix
// the CTA walks its block columns left to right (width NB = 32 or 64); the
// current block column (n rows x NB, fp32) lives in shared memory:
//
//   for block column j:
//     load it from global
//     for k < j:  U_kj = L_kk^-1 A_kj           (rows of block k; ib = 8
//                                                 chunks, FP32)
//                 A[rows >= NB(k+1), j] -= L_k U_kj
//                                                 (tcgen05, fp16 operands,
//                                                 fp32 accumulate in TMEM;
//                                                 or FP32 fma chains)
//     factor rows >= NB j of block column j      (ib = 8 chunks, FP32)
//     store it back
//
// Every element receives the same operations in the same order as the
// right-looking algorithm with outer block NB and inner block 8
// (src/lu_nopiv.hxx:130-197, src/lu_nopiv_inner_rl.hxx:104-196): outer
// updates from blocks k = 0, 1, ... one K = NB product each (acc from 0,
// subtracted once), then the inner elimination of its own block.  Only the
// schedule is left-looking, so with FP32 outer updates the factors equal the
// right-looking CPU restatement bit for bit; with fp16 operands only the
// tensor core's accumulation order differs.
//
// Inner elimination: the 8x8 diagonal tile (1/d correctly rounded, a
// multiply, fused a - l*u), the L rows below (row * 1/d, fused updates), the
// U columns right of it (forward substitution) and a rank-8 update
// accumulated acc = fma(l, u, acc) then subtracted (src/lu_nopiv.cu:105-326).
// Rows are owned by threads (row p by thread p mod 256), so each 8-column
// step costs one CTA barrier: the warp owning the tile's rows factors the
// tile and the U strip, then every thread eliminates and updates its own
// rows.
#include "common.cuh"
#include "kernels.cuh"
#include "panel_rows.cuh"
#include "sm100.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <new>
#include <numeric>
#include <vector>

namespace lub {
namespace {

using namespace sm100;
using rows::load8;

constexpr int kT = 256;                 // threads per CTA
constexpr int kWarps = kT / 32;
constexpr int kTileM = 128;             // rows per tensor-core tile
constexpr int kAStage = kTileM * 128;   // fp16 K-major tile, 128-byte rows
constexpr int kAOff = 0;                // 2 A stages (or one fp32 L tile)
constexpr int kBOff = 2 * kAStage;      // B operand (fp16) or U (fp32)
constexpr int kLOff = kBOff + 64 * 64 * 4;
constexpr int kLDT = 68;                // L_kk, row-major, row stride
constexpr int kUOff = kLOff + 64 * kLDT * 4;  // 2 x (8 x 64) substituted chunk rows
constexpr int kCOff = kUOff + 2 * 8 * 64 * 4;
constexpr int kTmemCols = 128;          // two 128 x 64 fp32 accumulators
constexpr uint32_t kIdesc = make_idesc(0, 0, kTileM, 64);  // fp16, M128 N64

enum : int { kErrBatchMma = 11 };

struct Misc {
  uint64_t bar[2];     // MMA of stage b done
  uint64_t ld[2];      // stage b's operand image landed
  uint32_t tmem;
  int item;
  int bad;
  int abort;
  float inv[2][8];
};

struct BatchArgs {
  float* const* ptrs;
  const int32_t* n;
  const int32_t* lda;     // may be null: lda = n
  int32_t* info;
  const int32_t* order;   // work list (matrix indices)
  const uint8_t* cfg;     // per work item: bit 0 tensor-core outer updates, bit 1 NB = 32
  int32_t count;
  int32_t* counter;       // zeroed before the launch
  int* err;
  int ldc;                // leading dimension of the block column in shared memory
  int use_tc;             // any tensor-core item: allocate TMEM
  uint8_t* img;           // per CTA: fp16 operand images of the factored L
                          // columns (img_bytes each), tensor-core items
  int64_t img_bytes;
};

// Bytes of the L operand images of one matrix (all its block columns but
// the last): per block column, one 16 KB image per 128-row tile of the rows
// below it.
__host__ __device__ inline int64_t img_tiles_before(int n, int NB, int j) {
  int64_t t = 0;
  for (int i = 0; i < j; ++i) {
    const int rows = n - (i + 1) * NB;
    if (rows > 0) t += (rows + kTileM - 1) / kTileM;
  }
  return t;
}

size_t smem_bytes_for(int nmax) {
  const int ldc = ((nmax + 3) / 4) * 4 + 4;
  return 1024 + (size_t)kCOff + (size_t)ldc * 64 * 4 + sizeof(Misc) + 16;
}

// ---------------------------------------------------------------------------
// Asynchronous copy of a rows x cols column-major block from global (ld gld)
// into shared memory at dst(r, c); 16-byte copies when both sides allow
// (vec: source 16-byte aligned, gld and rows' starts multiples of 4), so the
// whole block is in flight at once instead of one load latency per element.
template <typename DstIdx>
__device__ __forceinline__ void async_block(const float* src, int64_t gld, int rows,
                                            int cols, bool vec, DstIdx dst) {
  const int tid = threadIdx.x;
  if (vec) {
    const int r4 = rows >> 2;
    for (int idx = tid; idx < r4 * cols; idx += kT) {
      const int c = idx / r4, r = 4 * (idx - c * r4);
      cp_async16(dst(r, c), src + r + (int64_t)c * gld);
    }
    const int rt = rows & 3;
    for (int idx = tid; idx < rt * cols; idx += kT) {
      const int c = idx / rt, r = 4 * r4 + (idx - c * rt);
      cp_async4(dst(r, c), src + r + (int64_t)c * gld);
    }
  } else {
    for (int idx = tid; idx < rows * cols; idx += kT) {
      const int c = idx / rows, r = idx - c * rows;
      cp_async4(dst(r, c), src + r + (int64_t)c * gld);
    }
  }
  cp_async_wait_all();
}

// Shared (ld sld) -> global (ld gld) copy of a rows x cols column-major block.
__device__ __forceinline__ void store_block(float* dst, int64_t gld, int rows, int cols,
                                            bool vec, const float* src, int sld) {
  const int tid = threadIdx.x;
  if (vec) {
    const int r4 = rows >> 2;
    for (int idx = tid; idx < r4 * cols; idx += kT) {
      const int c = idx / r4, r = 4 * (idx - c * r4);
      *reinterpret_cast<float4*>(dst + r + (int64_t)c * gld) =
          *reinterpret_cast<const float4*>(src + r + c * sld);
    }
    const int rt = rows & 3;
    for (int idx = tid; idx < rt * cols; idx += kT) {
      const int c = idx / rt, r = 4 * r4 + (idx - c * rt);
      dst[r + (int64_t)c * gld] = src[r + c * sld];
    }
  } else {
    for (int idx = tid; idx < rows * cols; idx += kT) {
      const int c = idx / rows, r = idx - c * rows;
      dst[r + (int64_t)c * gld] = src[r + c * sld];
    }
  }
}

// ---------------------------------------------------------------------------
// U_kj = L_kk^-1 A_kj for rows [r0, r0 + NB) of the block column (wj <= 64
// columns), in 8-row chunks: forward substitution inside chunk q, then a
// rank-8 update of the later chunks.  Warp s owns chunk s (8 rows) of
// columns lane and lane + 32, so every L_kk read is a warp-wide broadcast;
// the substituted chunk is handed to the other warps through shared memory
// (double-buffered, one CTA barrier per chunk).  Also writes the B operand.
// Lt: L_kk row-major (row stride kLDT).
__device__ __forceinline__ void trsm_block(float* C, int ldc, const float* Lt,
                                           float* ustage, int r0, int NB, int wj,
                                           bool tc, uint8_t* sB) {
  const int s = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nch = NB >> 3;
  const bool mine = s < nch;
  const bool a0 = mine && lane < wj, a1 = mine && lane + 32 < wj;
  float v0[8], v1[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    v0[i] = a0 ? C[(r0 + 8 * s + i) + lane * ldc] : 0.0f;
    v1[i] = a1 ? C[(r0 + 8 * s + i) + (lane + 32) * ldc] : 0.0f;
  }
#pragma unroll 1
  for (int q = 0; q < nch; ++q) {
    float* us = ustage + (q & 1) * 512;
    if (s == q) {
#pragma unroll
      for (int i = 1; i < 8; ++i) {
        float l[8];
        load8(Lt + (8 * q + i) * kLDT + 8 * q, l);
#pragma unroll
        for (int kk = 0; kk < 8; ++kk) {
          if (kk < i) {
            v0[i] = __fmaf_rn(-l[kk], v0[kk], v0[i]);
            v1[i] = __fmaf_rn(-l[kk], v1[kk], v1[i]);
          }
        }
      }
      if (q + 1 < nch) {
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          us[i * 64 + lane] = v0[i];
          us[i * 64 + lane + 32] = v1[i];
        }
      }
    }
    if (q + 1 == nch) break;
    __syncthreads();
    if (mine && s > q) {
      float u0[8], u1[8];
#pragma unroll
      for (int kk = 0; kk < 8; ++kk) {
        u0[kk] = us[kk * 64 + lane];
        u1[kk] = us[kk * 64 + lane + 32];
      }
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        float l[8];
        load8(Lt + (8 * s + i) * kLDT + 8 * q, l);
        float acc0 = 0.0f, acc1 = 0.0f;
#pragma unroll
        for (int kk = 0; kk < 8; ++kk) {
          acc0 = __fmaf_rn(l[kk], u0[kk], acc0);
          acc1 = __fmaf_rn(l[kk], u1[kk], acc1);
        }
        v0[i] = __fsub_rn(v0[i], acc0);
        v1[i] = __fsub_rn(v1[i], acc1);
      }
    }
  }
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    if (a0) C[(r0 + 8 * s + i) + lane * ldc] = v0[i];
    if (a1) C[(r0 + 8 * s + i) + (lane + 32) * ldc] = v1[i];
  }
  if (tc) {
    // B row c (N index), 16-byte chunk s (K = 8s .. 8s+7), 128-byte swizzle
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int c = lane + 32 * h;
      const bool act = h ? a1 : a0;
      const float* v = h ? v1 : v0;
      if (!mine) continue;
      uint4 pk = make_uint4(0, 0, 0, 0);
      if (act) {
        __half2 h0 = __floats2half2_rn(v[0], v[1]);
        __half2 h1 = __floats2half2_rn(v[2], v[3]);
        __half2 h2 = __floats2half2_rn(v[4], v[5]);
        __half2 h3 = __floats2half2_rn(v[6], v[7]);
        pk.x = *reinterpret_cast<uint32_t*>(&h0);
        pk.y = *reinterpret_cast<uint32_t*>(&h1);
        pk.z = *reinterpret_cast<uint32_t*>(&h2);
        pk.w = *reinterpret_cast<uint32_t*>(&h3);
      }
      *reinterpret_cast<uint4*>(sB + c * 128 + ((s ^ (c & 7)) << 4)) = pk;
    }
  } else if (mine) {
    float* Bf = reinterpret_cast<float*>(sB);  // U row-major [kk][64]
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      Bf[(8 * s + i) * 64 + lane] = a0 ? v0[i] : 0.0f;
      Bf[(8 * s + i) * 64 + lane + 32] = a1 ? v1[i] : 0.0f;
    }
  }
}

// ---------------------------------------------------------------------------
// FP32 outer update: rows [r1, n) of the block column -= L[rows, r0:r0+NB] U
// (U row-major fp32 in sB), acc over K from 0 in order, subtracted once.
__device__ __forceinline__ void outer_fp32(float* C, int ldc, const float* A,
                                           int64_t lda, int n, int r0, int NB,
                                           int wj, uint8_t* sA, const uint8_t* sB) {
  const int tid = threadIdx.x;
  const int r1 = r0 + NB;
  float* Ls = reinterpret_cast<float*>(sA);         // [NB][128]
  const float* Bf = reinterpret_cast<const float*>(sB);  // [NB][64]
  const int rb = 4 * (tid & 31), cb = 8 * (tid >> 5);
#pragma unroll 1
  for (int m0 = r1; m0 < n; m0 += kTileM) {
    const int rows = min(kTileM, n - m0);
    if (rows < kTileM) {
      for (int idx = tid; idx < (kTileM - rows) * NB; idx += kT) {
        const int kk = idx / (kTileM - rows), m = rows + idx % (kTileM - rows);
        Ls[m + kk * kTileM] = 0.0f;
      }
    }
    async_block(A + m0 + (int64_t)r0 * lda, lda, rows, NB, false,
                [&](int r, int c) { return &Ls[r + c * kTileM]; });
    __syncthreads();
    float acc[4][8];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int jj = 0; jj < 8; ++jj) acc[i][jj] = 0.0f;
#pragma unroll 4
    for (int kk = 0; kk < NB; ++kk) {
      const float4 l4 = *reinterpret_cast<const float4*>(&Ls[rb + kk * kTileM]);
      const float4 ua = *reinterpret_cast<const float4*>(&Bf[kk * 64 + cb]);
      const float4 ub = *reinterpret_cast<const float4*>(&Bf[kk * 64 + cb + 4]);
      const float l[4] = {l4.x, l4.y, l4.z, l4.w};
      const float u[8] = {ua.x, ua.y, ua.z, ua.w, ub.x, ub.y, ub.z, ub.w};
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int jj = 0; jj < 8; ++jj) acc[i][jj] = __fmaf_rn(l[i], u[jj], acc[i][jj]);
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int row = m0 + rb + i;
      if (row < n) {
#pragma unroll
        for (int jj = 0; jj < 8; ++jj)
          if (cb + jj < wj) {
            float* p = &C[row + (cb + jj) * ldc];
            *p = __fsub_rn(*p, acc[i][jj]);
          }
      }
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Tensor-core outer update: per 128-row tile, stage fp16(L) K-major with the
// 128-byte swizzle, one thread issues NB/16 MMAs (M128 N64 K16) into one of
// two TMEM accumulators, and the epilogue of the previous tile (all eight
// warps: lane quarter warp%4, 32 columns each) subtracts its product from
// the block column while the next MMAs run.
// Epilogue of one tile, its MMAs known complete: all eight warps (lane
// quarter warp % 4, 32 columns each) subtract the accumulator from the
// block column.
__device__ __forceinline__ void tc_epilogue_read(float* C, int ldc, int n, int wj, int m0,
                                                 int b, uint32_t tmem) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncwarp();
  tc_fence_after();
  const int quarter = warp & 3, half = warp >> 2;
  float pv[32];
  tmem_ld32(tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(b * 64 + half * 32), pv);
  tmem_ld_wait();
  const int row = m0 + quarter * 32 + lane;
  if (row < n) {
#pragma unroll
    for (int cc = 0; cc < 32; ++cc) {
      const int c = half * 32 + cc;
      if (c < wj) {
        float* p = &C[row + c * ldc];
        *p = __fsub_rn(*p, pv[cc]);
      }
    }
  }
  tc_fence_before();
}

// Tensor-core outer update from the operand images of block column k
// (written once, when k was factored): per 128-row tile one 16 KB bulk copy
// into a stage (two stages, the next tile's copy issued as soon as its
// stage is free), NB/16 MMAs into one of two TMEM accumulators, and the
// epilogue of the previous tile (all eight warps) under the MMAs.
struct TcState {
  uint32_t phase[2];
  uint32_t ldph[2];
};

// The first two tiles' copies, issued (thread 0) before the U_kj solve so
// that they land while it runs (the stages are free during the solve).
__device__ __forceinline__ void outer_tc_prefetch(const uint8_t* img, int n, int r0, int NB,
                                                  uint8_t* sA, Misc* ms) {
  const int ntiles = (n - r0 - NB + kTileM - 1) / kTileM;
  if (threadIdx.x == 0) {
    fence_proxy_async_smem();  // earlier generic accesses to the stages first
    for (int t = 0; t < 2 && t < ntiles; ++t) {
      mbar_arrive_expect_tx(&ms->ld[t], kAStage);
      bulk_load(sA + t * kAStage, img + (size_t)t * kAStage, kAStage, &ms->ld[t]);
    }
  }
}

__device__ __forceinline__ void outer_tc(float* C, int ldc, const uint8_t* img, int n,
                                         int r0, int NB, int wj, uint8_t* sA,
                                         const uint8_t* sB, uint32_t tmem, Misc* ms,
                                         TcState& st, int* err) {
  const int tid = threadIdx.x;
  const int r1 = r0 + NB;
  const int ntiles = (n - r1 + kTileM - 1) / kTileM;
#pragma unroll 1
  for (int t = 0; t < ntiles; ++t) {
    const int b = t & 1;
    const int m0 = r1 + t * kTileM;
    uint8_t* sa = sA + b * kAStage;
    tc_fence_before();
    __syncthreads();  // accumulator b read out by the epilogue of tile t - 2
    if (tid == 0) {
      tc_fence_after();
      if (!mbar_wait(&ms->ld[b], st.ldph[b], err, kErrBatchMma)) ms->abort = 1;
      const uint32_t a0 = smem_u32(sa), b0 = smem_u32(sB);
      for (int kq = 0; kq < NB / 16; ++kq)
        mma_f16(tmem + b * 64, sw128_kmajor_desc(a0 + kq * 32),
                sw128_kmajor_desc(b0 + kq * 32), kIdesc, kq > 0 ? 1u : 0u);
      mma_commit(&ms->bar[b]);
    }
    st.ldph[b] ^= 1u;
    if (t > 0) {
      const int bp = b ^ 1;
      const bool ok = mbar_wait(&ms->bar[bp], st.phase[bp], err, kErrBatchMma);
      st.phase[bp] ^= 1u;
      if (!ok) ms->abort = 1;
      // stage bp is free: the copy of tile t + 1 goes in now
      if (tid == 0 && t + 1 < ntiles) {
        mbar_arrive_expect_tx(&ms->ld[bp], kAStage);
        bulk_load(sA + bp * kAStage, img + (size_t)(t + 1) * kAStage, kAStage, &ms->ld[bp]);
      }
      tc_epilogue_read(C, ldc, n, wj, m0 - kTileM, bp, tmem);
    }
  }
  if (ntiles > 0) {
    const int bl = (ntiles - 1) & 1;
    const bool ok = mbar_wait(&ms->bar[bl], st.phase[bl], err, kErrBatchMma);
    st.phase[bl] ^= 1u;
    if (!ok) ms->abort = 1;
    tc_epilogue_read(C, ldc, n, wj, r1 + (ntiles - 1) * kTileM, bl, tmem);
  }
  tc_fence_before();
  __syncthreads();
}

// The operand images of block column c0 / NB, from the factored block
// column in shared memory (global row r, local column c at C[r + c ldc]):
// rows [c0 + NB, n) of its NB columns, fp16, one
// 128-row K-major tile with the 128-byte swizzle per 16 KB (rows past n
// zero), exactly what a stage of the outer update holds.
__device__ __forceinline__ void write_images(const float* C, int ldc, int n, int c0, int NB,
                                             uint8_t* img) {
  const int r1 = c0 + NB;
  const int ntiles = (n - r1 + kTileM - 1) / kTileM;
  const int nch = NB >> 3;
  for (int idx = threadIdx.x; idx < ntiles * kTileM * nch; idx += kT) {
    const int ch = idx % nch, rem = idx / nch;
    const int m = rem % kTileM, t = rem / kTileM;
    const int gr = r1 + t * kTileM + m;
    uint4 pk = make_uint4(0, 0, 0, 0);
    if (gr < n) {
      float x[8];
#pragma unroll
      for (int e = 0; e < 8; ++e) x[e] = C[gr + (8 * ch + e) * ldc];  // local columns
      __half2 h0 = __floats2half2_rn(x[0], x[1]);
      __half2 h1 = __floats2half2_rn(x[2], x[3]);
      __half2 h2 = __floats2half2_rn(x[4], x[5]);
      __half2 h3 = __floats2half2_rn(x[6], x[7]);
      pk.x = *reinterpret_cast<uint32_t*>(&h0);
      pk.y = *reinterpret_cast<uint32_t*>(&h1);
      pk.z = *reinterpret_cast<uint32_t*>(&h2);
      pk.w = *reinterpret_cast<uint32_t*>(&h3);
    }
    *reinterpret_cast<uint4*>(img + (size_t)t * kAStage + m * 128 + ((ch ^ (m & 7)) << 4)) = pk;
  }
}

// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kT, 1) batch_lu_kernel(BatchArgs a) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* sm = reinterpret_cast<uint8_t*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint8_t* sA = sm + kAOff;
  uint8_t* sB = sm + kBOff;
  float* Lkk = reinterpret_cast<float*>(sm + kLOff);
  float* ustage = reinterpret_cast<float*>(sm + kUOff);
  float* C = reinterpret_cast<float*>(sm + kCOff);
  Misc* ms = reinterpret_cast<Misc*>(sm + kCOff + (size_t)a.ldc * 64 * 4);
  const int tid = threadIdx.x;
  const int ldc = a.ldc;

  if (tid == 0) {
    mbar_init(&ms->bar[0], 1);
    mbar_init(&ms->bar[1], 1);
    mbar_init(&ms->ld[0], 1);
    mbar_init(&ms->ld[1], 1);
    fence_barrier_init();
    ms->abort = 0;
  }
  if (a.use_tc && (tid >> 5) == 0) tmem_alloc(&ms->tmem, kTmemCols);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = a.use_tc ? ms->tmem : 0u;
  TcState st;
  st.phase[0] = st.phase[1] = 0u;
  st.ldph[0] = st.ldph[1] = 0u;
  uint8_t* img = a.img ? a.img + (size_t)blockIdx.x * (size_t)a.img_bytes : nullptr;

#pragma unroll 1
  for (;;) {
    if (tid == 0) {
      ms->item = atomicAdd(a.counter, 1);
      ms->bad = kNoBadPivot;
    }
    __syncthreads();
    const int it = ms->item;
    if (it >= a.count || ms->abort) break;
    const int mat = a.order[it];
    const int cfg = a.cfg[it];
    const bool tc = (cfg & 1) != 0 && a.use_tc;
    const int NB = (cfg & 2) ? 32 : 64;
    const int n = a.n[mat];
    const int64_t lda = a.lda ? (int64_t)a.lda[mat] : (int64_t)n;
    float* A = a.ptrs[mat];
    const bool vec = ((reinterpret_cast<uintptr_t>(A) & 15) == 0) && (lda % 4 == 0);
    const int nblk = (n + NB - 1) / NB;
#pragma unroll 1
    for (int j = 0; j < nblk && !ms->abort; ++j) {
      const int c0 = j * NB;
      const int wj = min(NB, n - c0);
      async_block(A + (int64_t)c0 * lda, lda, n, wj, vec,
                  [&](int r, int c) { return &C[r + c * ldc]; });
      __syncthreads();
#pragma unroll 1
      for (int k = 0; k < j; ++k) {
        const int r0 = k * NB;
        if (tc && r0 + NB < n)
          outer_tc_prefetch(img + (size_t)img_tiles_before(n, NB, k) * kAStage, n, r0, NB, sA,
                            ms);
        async_block(A + r0 + (int64_t)r0 * lda, lda, NB, NB, false,
                    [&](int r, int c) { return &Lkk[r * kLDT + c]; });
        __syncthreads();
        trsm_block(C, ldc, Lkk, ustage, r0, NB, wj, tc, sB);
        if (tc) fence_proxy_async_smem();
        __syncthreads();
        if (r0 + NB < n) {
          if (tc)
            outer_tc(C, ldc, img + (size_t)img_tiles_before(n, NB, k) * kAStage, n, r0, NB, wj,
                     sA, sB, tmem, ms, st, a.err);
          else outer_fp32(C, ldc, A, lda, n, r0, NB, wj, sA, sB);
        }
        if (ms->abort) break;
      }
      if (ms->abort) break;
      rows::panel_block<kT>(C, ldc, n, c0, wj, &ms->inv[0][0], &ms->bad, c0);
      store_block(A + (int64_t)c0 * lda, lda, n, wj, vec, C, ldc);
      // the later block columns' outer updates read this one's L rows as
      // fp16 operand images, by bulk copy
      if (tc && j + 1 < nblk) {
        write_images(C, ldc, n, c0, NB, img + (size_t)img_tiles_before(n, NB, j) * kAStage);
        fence_proxy_async_global();
      }
      __syncthreads();
    }
    if (tid == 0)
      a.info[mat] = ms->abort ? -1 : (ms->bad == kNoBadPivot ? 0 : ms->bad);
    __syncthreads();
  }

  tc_fence_before();
  __syncthreads();
  if (a.use_tc && (tid >> 5) == 0) {
    tc_fence_after();
    tmem_dealloc(tmem, kTmemCols);
  }
}

// ---------------------------------------------------------------------------
// host side

int bucket_of(int n) {
  int b = 0;
  while ((32 << b) <= n && b < LU_BATCH_BUCKETS - 1) ++b;
  return b;
}

uint8_t cfg_of(const lu_batch_tuning& t, int n) {
  const int b = bucket_of(n);
  uint8_t c = 0;
  if (t.outer[b] == LU_COMPUTE_TC32) c |= 1;
  if (t.nb[b] == 32) c |= 2;
  return c;
}

}  // namespace

}  // namespace lub

using namespace lub;

struct lu_batch_plan_t {
  int device = 0;
  int64_t batch = 0;
  int nmax = 0;
  std::vector<int32_t> h_n;
  std::vector<int32_t> h_order;
  lu_batch_tuning tuning{};
  int32_t* d_n = nullptr;
  int32_t* d_order = nullptr;
  uint8_t* d_cfg = nullptr;
  int32_t* d_counter = nullptr;  // [0] work counter, [1] error flag
  int ctas = 0;
  size_t smem = 0;
  bool use_tc = false;
  uint8_t* d_img = nullptr;  // per CTA: operand images (tensor-core items)
  int64_t img_bytes = 0;
  size_t img_alloc = 0;
  lu_opts opts{};
};

namespace lub {
int64_t batch_plan_size(const lu_batch_plan_t* p) { return p->batch; }
const int32_t* batch_plan_dev_n(const lu_batch_plan_t* p) { return p->d_n; }
int batch_plan_nmax(const lu_batch_plan_t* p) { return p->nmax; }
}  // namespace lub

struct lu_batch_graph_t {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

namespace {

lu_status upload_cfg(lu_batch_plan_t* p) {
  std::vector<uint8_t> cfg(p->batch);
  p->use_tc = false;
  for (int64_t i = 0; i < p->batch; ++i) {
    const int n = p->h_n[p->h_order[i]];
    cfg[i] = cfg_of(p->tuning, n);
    if ((cfg[i] & 1) && n > ((cfg[i] & 2) ? 32 : 64)) p->use_tc = true;
  }
  LUB_CUDA_TRY(cudaMemcpy(p->d_cfg, cfg.data(), cfg.size(), cudaMemcpyHostToDevice));
  p->smem = smem_bytes_for(p->nmax);
  int sms = 0;
  LUB_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, p->device));
  LUB_CUDA_TRY(set_smem_limit((const void*)batch_lu_kernel, p->smem));
  int per_sm = 0;
  LUB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      &per_sm, batch_lu_kernel, kT, p->smem));
  if (per_sm < 1) return LU_ERR_UNSUPPORTED;
  p->ctas = (int)std::min<int64_t>((int64_t)sms * per_sm, p->batch);
  // operand images: the largest matrix's, at the block width needing most
  p->img_bytes = 0;
  if (p->use_tc) {
    const int nm = p->nmax;
    for (int NB : {32, 64})
      p->img_bytes = std::max<int64_t>(p->img_bytes,
                                       img_tiles_before(nm, NB, (nm + NB - 1) / NB) * kAStage);
    const size_t need = (size_t)p->ctas * (size_t)p->img_bytes;
    if (need > p->img_alloc) {
      cudaFree(p->d_img);
      p->d_img = nullptr;
      p->img_alloc = 0;
      if (cudaMalloc(&p->d_img, need) != cudaSuccess) return LU_ERR_ALLOC;
      p->img_alloc = need;
    }
  }
  return LU_SUCCESS;
}

void default_tuning(const lu_opts* o, lu_batch_tuning* t) {
  const bool tcq = o->outer_update == LU_COMPUTE_TC32;
  for (int b = 0; b < LU_BATCH_BUCKETS; ++b) {
    t->nb[b] = (o->nb == 32 || o->nb == 64) ? o->nb : 64;
    t->outer[b] = tcq ? LU_COMPUTE_TC32 : LU_COMPUTE_FP32;
  }
}

lu_status check_tuning(const lu_batch_tuning* t) {
  for (int b = 0; b < LU_BATCH_BUCKETS; ++b) {
    if (t->nb[b] != 32 && t->nb[b] != 64) return LU_ERR_INVALID_ARG;
    if (t->outer[b] != LU_COMPUTE_FP32 && t->outer[b] != LU_COMPUTE_TC32)
      return LU_ERR_UNSUPPORTED;
  }
  return LU_SUCCESS;
}

lu_status launch_plan(const lu_batch_plan_t* p, cudaStream_t st, float* const* d_ptrs,
                      const int32_t* d_lda, int32_t* d_info, const int32_t* order,
                      const uint8_t* cfg, int64_t count) {
  LUB_CUDA_TRY(cudaMemsetAsync(p->d_counter, 0, 2 * sizeof(int32_t), st));
  BatchArgs a;
  a.ptrs = d_ptrs;
  a.n = p->d_n;
  a.lda = d_lda;
  a.info = d_info;
  a.order = order;
  a.cfg = cfg;
  a.count = (int32_t)count;
  a.counter = p->d_counter;
  a.err = p->d_counter + 1;
  a.ldc = ((p->nmax + 3) / 4) * 4 + 4;
  a.use_tc = p->use_tc ? 1 : 0;
  a.img = p->use_tc ? p->d_img : nullptr;
  a.img_bytes = p->img_bytes;
  const int ctas = (int)std::min<int64_t>(p->ctas, count);
  batch_lu_kernel<<<ctas, kT, p->smem, st>>>(a);
  LUB_LAUNCH_CHECK();
  return LU_SUCCESS;
}

}  // namespace

extern "C" {

LU_API lu_status lu_batch_plan_create(const lu_opts* opts, int64_t batch,
                                      const int32_t* h_n, const lu_batch_tuning* tuning,
                                      lu_batch_plan* plan) {
  if (!opts || !plan || batch < 0 || (batch > 0 && !h_n)) return LU_ERR_INVALID_ARG;
  *plan = nullptr;
  if (opts->inner_update != LU_COMPUTE_FP32) return LU_ERR_UNSUPPORTED;
  if (opts->outer_update != LU_COMPUTE_FP32 && opts->outer_update != LU_COMPUTE_TC32)
    return LU_ERR_UNSUPPORTED;
  if (opts->nb != 0 && opts->nb != 32 && opts->nb != 64) return LU_ERR_INVALID_ARG;
  if (batch > INT32_MAX) return LU_ERR_INVALID_ARG;
  for (int64_t i = 0; i < batch; ++i)
    if (h_n[i] < 1 || h_n[i] > LU_BATCH_MAX_N) return LU_ERR_INVALID_ARG;
  lu_batch_tuning t;
  if (tuning) {
    t = *tuning;
    LUB_TRY(check_tuning(&t));
  } else {
    default_tuning(opts, &t);
  }
  lu_batch_plan_t* p = new (std::nothrow) lu_batch_plan_t;
  if (!p) return LU_ERR_ALLOC;
  p->batch = batch;
  p->tuning = t;
  p->opts = *opts;
  p->h_n.assign(h_n, h_n + batch);
  p->h_order.resize(batch);
  std::iota(p->h_order.begin(), p->h_order.end(), 0);
  // decreasing size: the largest factorizations start first
  std::stable_sort(p->h_order.begin(), p->h_order.end(),
                   [&](int32_t x, int32_t y) { return p->h_n[x] > p->h_n[y]; });
  p->nmax = batch > 0 ? p->h_n[p->h_order[0]] : 1;
  lu_status s = LU_SUCCESS;
  if (cudaGetDevice(&p->device) != cudaSuccess) s = LU_ERR_NO_DEVICE;
  const size_t nb = std::max<int64_t>(batch, 1);
  if (s == LU_SUCCESS &&
      (cudaMalloc(&p->d_n, nb * 4) != cudaSuccess ||
       cudaMalloc(&p->d_order, nb * 4) != cudaSuccess ||
       cudaMalloc(&p->d_cfg, nb) != cudaSuccess ||
       cudaMalloc(&p->d_counter, 2 * sizeof(int32_t)) != cudaSuccess))
    s = LU_ERR_ALLOC;
  if (s == LU_SUCCESS && batch > 0 &&
      (cudaMemcpy(p->d_n, p->h_n.data(), batch * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
       cudaMemcpy(p->d_order, p->h_order.data(), batch * 4, cudaMemcpyHostToDevice) !=
           cudaSuccess))
    s = LU_ERR_CUDA;
  if (s == LU_SUCCESS && batch > 0) s = upload_cfg(p);
  if (s != LU_SUCCESS) {
    lu_batch_plan_destroy(p);
    return s;
  }
  *plan = p;
  return LU_SUCCESS;
}

LU_API void lu_batch_plan_destroy(lu_batch_plan plan) {
  if (!plan) return;
  cudaFree(plan->d_n);
  cudaFree(plan->d_order);
  cudaFree(plan->d_cfg);
  cudaFree(plan->d_counter);
  cudaFree(plan->d_img);
  delete plan;
}

LU_API lu_status lu_batch_plan_tuning(lu_batch_plan plan, lu_batch_tuning* out) {
  if (!plan || !out) return LU_ERR_INVALID_ARG;
  *out = plan->tuning;
  return LU_SUCCESS;
}

LU_API lu_status lu_batch_plan_set_tuning(lu_batch_plan plan, const lu_batch_tuning* t) {
  if (!plan || !t) return LU_ERR_INVALID_ARG;
  LUB_TRY(check_tuning(t));
  plan->tuning = *t;
  if (plan->batch == 0) return LU_SUCCESS;
  return upload_cfg(plan);
}

LU_API lu_status lu_batch_c(lu_batch_plan plan, lu_stream_t stream, float* const* d_ptrs,
                            const int32_t* d_lda, int32_t* d_info) {
  if (!plan) return LU_ERR_INVALID_ARG;
  if (plan->batch == 0) return LU_SUCCESS;
  if (!d_ptrs || !d_info) return LU_ERR_INVALID_ARG;
  return launch_plan(plan, (cudaStream_t)stream, d_ptrs, d_lda, d_info, plan->d_order,
                     plan->d_cfg, plan->batch);
}

LU_API lu_status lu_batch_autotune(lu_batch_plan plan, lu_stream_t stream, int reps,
                                   lu_batch_tuning* out) {
  if (!plan || reps < 1) return LU_ERR_INVALID_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  // candidate block widths per bucket, at the plan's outer precision
  const int outer = plan->opts.outer_update;
  const int widths[2] = {32, 64};
  lu_batch_tuning best = plan->tuning;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  LUB_CUDA_TRY(cudaEventCreate(&e0));
  LUB_CUDA_TRY(cudaEventCreate(&e1));
  lu_status s = LU_SUCCESS;
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, plan->device);
  for (int b = 0; b < LU_BATCH_BUCKETS && s == LU_SUCCESS; ++b) {
    // the bucket's sizes, sampled evenly down to at most 4 matrices per SM
    std::vector<int32_t> sz;
    for (int32_t i : plan->h_order)
      if (bucket_of(plan->h_n[i]) == b) sz.push_back(plan->h_n[i]);
    if (sz.empty()) continue;
    const size_t cap = (size_t)4 * sms;
    if (sz.size() > cap) {
      std::vector<int32_t> smp(cap);
      for (size_t i = 0; i < cap; ++i) smp[i] = sz[i * sz.size() / cap];
      sz.swap(smp);
    }
    const int64_t cnt = (int64_t)sz.size();
    std::vector<int64_t> off(cnt + 1, 0);
    for (int64_t i = 0; i < cnt; ++i) off[i + 1] = off[i] + (int64_t)sz[i] * sz[i];
    float* buf = nullptr;
    float* src = nullptr;
    float** dptr = nullptr;
    int32_t* dn = nullptr;
    int32_t* dinfo = nullptr;
    if (cudaMalloc(&buf, off[cnt] * 4) != cudaSuccess ||
        cudaMalloc(&src, off[cnt] * 4) != cudaSuccess ||
        cudaMalloc(&dptr, cnt * sizeof(float*)) != cudaSuccess ||
        cudaMalloc(&dn, cnt * 4) != cudaSuccess || cudaMalloc(&dinfo, cnt * 4) != cudaSuccess)
      s = LU_ERR_ALLOC;
    std::vector<float*> hp(cnt);
    for (int64_t i = 0; i < cnt; ++i) hp[i] = src + off[i];
    if (s == LU_SUCCESS &&
        (cudaMemcpy(dptr, hp.data(), cnt * sizeof(float*), cudaMemcpyHostToDevice) != cudaSuccess ||
         cudaMemcpy(dn, sz.data(), cnt * 4, cudaMemcpyHostToDevice) != cudaSuccess))
      s = LU_ERR_CUDA;
    if (s == LU_SUCCESS) s = launch_gen_batch(st, cnt, dptr, dn, nullptr, 11 + b, 0, 1.5);
    for (int64_t i = 0; i < cnt; ++i) hp[i] = buf + off[i];
    if (s == LU_SUCCESS &&
        cudaMemcpy(dptr, hp.data(), cnt * sizeof(float*), cudaMemcpyHostToDevice) != cudaSuccess)
      s = LU_ERR_CUDA;
    float best_ms = INFINITY;
    for (int w = 0; w < 2 && s == LU_SUCCESS; ++w) {
      lu_batch_tuning t = plan->tuning;
      for (int q = 0; q < LU_BATCH_BUCKETS; ++q) {
        t.nb[q] = widths[w];
        t.outer[q] = outer;
      }
      lu_batch_plan sub = nullptr;
      s = lu_batch_plan_create(&plan->opts, cnt, sz.data(), &t, &sub);
      if (s != LU_SUCCESS) break;
      std::vector<float> times;
      for (int r = 0; r < reps + 1 && s == LU_SUCCESS; ++r) {
        if (cudaMemcpyAsync(buf, src, off[cnt] * 4, cudaMemcpyDeviceToDevice, st) != cudaSuccess ||
            cudaEventRecord(e0, st) != cudaSuccess) {
          s = LU_ERR_CUDA;
          break;
        }
        s = lu_batch_c(sub, stream, dptr, nullptr, dinfo);
        float ms = 0.0f;
        if (s == LU_SUCCESS &&
            (cudaEventRecord(e1, st) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
             cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess))
          s = LU_ERR_CUDA;
        if (r > 0) times.push_back(ms);  // the first run warms up
      }
      lu_batch_plan_destroy(sub);
      if (s != LU_SUCCESS || times.empty()) break;
      std::sort(times.begin(), times.end());
      const float med = times[times.size() / 2];
      if (med < best_ms) {
        best_ms = med;
        best.nb[b] = widths[w];
        best.outer[b] = outer;
      }
    }
    cudaFree(buf);
    cudaFree(src);
    cudaFree(dptr);
    cudaFree(dn);
    cudaFree(dinfo);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (s != LU_SUCCESS) return s;
  plan->tuning = best;
  if (plan->batch > 0) LUB_TRY(upload_cfg(plan));
  if (out) *out = best;
  return LU_SUCCESS;
}

LU_API lu_status lu_batch_graph_create(lu_batch_plan plan, lu_stream_t stream,
                                       float* const* d_ptrs, const int32_t* d_lda,
                                       int32_t* d_info, lu_batch_graph* graph) {
  if (!plan || !graph) return LU_ERR_INVALID_ARG;
  *graph = nullptr;
  lu_batch_graph_t* g = new (std::nothrow) lu_batch_graph_t;
  if (!g) return LU_ERR_ALLOC;
  cudaStream_t st = (cudaStream_t)stream;
  lu_status s = LU_SUCCESS;
  if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    delete g;
    return LU_ERR_CUDA;
  }
  s = lu_batch_c(plan, stream, d_ptrs, d_lda, d_info);
  cudaGraph_t gr = nullptr;
  const cudaError_t e = cudaStreamEndCapture(st, &gr);
  if (s == LU_SUCCESS && e != cudaSuccess) s = LU_ERR_CUDA;
  if (s == LU_SUCCESS && cudaGraphInstantiate(&g->exec, gr, 0) != cudaSuccess) s = LU_ERR_CUDA;
  g->graph = gr;
  if (s != LU_SUCCESS) {
    lu_batch_graph_destroy(g);
    return s;
  }
  *graph = g;
  return LU_SUCCESS;
}

LU_API lu_status lu_batch_graph_launch(lu_batch_graph graph, lu_stream_t stream) {
  if (!graph || !graph->exec) return LU_ERR_INVALID_ARG;
  LUB_CUDA_TRY(cudaGraphLaunch(graph->exec, (cudaStream_t)stream));
  count_launch();
  return LU_SUCCESS;
}

LU_API void lu_batch_graph_destroy(lu_batch_graph graph) {
  if (!graph) return;
  if (graph->exec) cudaGraphExecDestroy(graph->exec);
  if (graph->graph) cudaGraphDestroy(graph->graph);
  delete graph;
}

}  // extern "C"
