// FP32 SIMT update C = alpha*A*B + beta*C for the FP32 plain path.
//
// Replaces the reference's cublasSgemm call (src/gemm.cu:17-35) used for the
// outer Schur update (src/lu_nopiv.hxx:185-192) and the K = 8 inner updates
// (src/lu_nopiv_inner_rl.hxx:155-190).  No tensor cores: the FP32 plain path
// must stay FP32-faithful.
//
// Accumulation order, per output element: acc = fma(A[i,t], B[t,j], acc) for
// t = 0..K-1 from acc = 0, then C = C - acc (alpha = -1, beta = 1).  With
// CHUNK8 the K range is consumed in blocks of 8 and C -= acc after every
// block, which is how the reference's sequence of rank-8 updates inside an
// outer block composes; this lets one launch apply several inner steps while
// every element still sees the reference's sequence.
//
// Tiling: 128 x 128 per CTA, 256 threads with an 8 x 8 register tile each
// (rows tx*4..+3 and 64+tx*4..+3, columns likewise), K staged 8 at a time
// through double-buffered shared memory.
#include "common.cuh"
#include "kernels.cuh"

namespace lub {
namespace {

constexpr int BM = 128, BN = 128, BK = 8, NT = 256;

template <bool CHUNK8, bool VEC>
__global__ void __launch_bounds__(NT)
sgemm_update_kernel(int64_t M, int64_t N, int64_t K, float alpha,
                    const float* __restrict__ A, int64_t lda,
                    const float* __restrict__ B, int64_t ldb, float beta,
                    float* __restrict__ C, int64_t ldc) {
  __shared__ __align__(16) float As[2][BK][BM];
  __shared__ __align__(16) float Bs[2][BK][BN];

  const int tid = threadIdx.x;
  const int tx = tid % 16, ty = tid / 16;
  const int64_t m0 = (int64_t)blockIdx.x * BM;
  const int64_t n0 = (int64_t)blockIdx.y * BN;

  // loader coordinates
  // A tile BM x BK: thread loads 4 consecutive rows of one column.
  const int a_col = tid / 32;         // 0..7
  const int a_row = (tid % 32) * 4;   // 0..124
  // B tile BK x BN: thread loads 4 consecutive k of one column.
  const int b_col = tid / 2;          // 0..127
  const int b_k = (tid % 2) * 4;      // 0 or 4

  float ra[4], rb[4];
  auto load_tiles = [&](int64_t k0) {
    const int64_t ak = k0 + a_col;
    const int64_t ar = m0 + a_row;
    if (VEC && ak < K && ar + 3 < M) {
      const float4 v = *reinterpret_cast<const float4*>(A + ar + ak * lda);
      ra[0] = v.x; ra[1] = v.y; ra[2] = v.z; ra[3] = v.w;
    } else {
#pragma unroll
      for (int i = 0; i < 4; ++i)
        ra[i] = (ak < K && ar + i < M) ? A[ar + i + ak * lda] : 0.0f;
    }
    const int64_t bc = n0 + b_col;
    const int64_t bk = k0 + b_k;
    if (VEC && bc < N && bk + 3 < K) {
      const float4 v = *reinterpret_cast<const float4*>(B + bk + bc * ldb);
      rb[0] = v.x; rb[1] = v.y; rb[2] = v.z; rb[3] = v.w;
    } else {
#pragma unroll
      for (int i = 0; i < 4; ++i)
        rb[i] = (bc < N && bk + i < K) ? B[bk + i + bc * ldb] : 0.0f;
    }
  };
  auto store_tiles = [&](int buf) {
    *reinterpret_cast<float4*>(&As[buf][a_col][a_row]) =
        make_float4(ra[0], ra[1], ra[2], ra[3]);
#pragma unroll
    for (int i = 0; i < 4; ++i) Bs[buf][b_k + i][b_col] = rb[i];
  };

  float acc[8][8];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[i][j] = 0.0f;

  // output coordinates of this thread
  auto row_of = [&](int i) -> int64_t {
    return m0 + (i < 4 ? tx * 4 + i : 64 + tx * 4 + (i - 4));
  };
  auto col_of = [&](int j) -> int64_t {
    return n0 + (j < 4 ? ty * 4 + j : 64 + ty * 4 + (j - 4));
  };

  float cr[CHUNK8 ? 8 : 1][CHUNK8 ? 8 : 1];
  if constexpr (CHUNK8) {
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const int64_t r = row_of(i), c = col_of(j);
        cr[i][j] = (r < M && c < N) ? C[r + c * ldc] : 0.0f;
      }
  }

  const int64_t nk = (K + BK - 1) / BK;
  load_tiles(0);
  store_tiles(0);
  __syncthreads();
  for (int64_t kt = 0; kt < nk; ++kt) {
    const int buf = (int)(kt & 1);
    if (kt + 1 < nk) load_tiles((kt + 1) * BK);
#pragma unroll
    for (int k = 0; k < BK; ++k) {
      float a[8], b[8];
      const float4 a0 = *reinterpret_cast<const float4*>(&As[buf][k][tx * 4]);
      const float4 a1 = *reinterpret_cast<const float4*>(&As[buf][k][64 + tx * 4]);
      const float4 b0 = *reinterpret_cast<const float4*>(&Bs[buf][k][ty * 4]);
      const float4 b1 = *reinterpret_cast<const float4*>(&Bs[buf][k][64 + ty * 4]);
      a[0] = a0.x; a[1] = a0.y; a[2] = a0.z; a[3] = a0.w;
      a[4] = a1.x; a[5] = a1.y; a[6] = a1.z; a[7] = a1.w;
      b[0] = b0.x; b[1] = b0.y; b[2] = b0.z; b[3] = b0.w;
      b[4] = b1.x; b[5] = b1.y; b[6] = b1.z; b[7] = b1.w;
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = __fmaf_rn(a[i], b[j], acc[i][j]);
    }
    if constexpr (CHUNK8) {
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          cr[i][j] = __fsub_rn(cr[i][j], acc[i][j]);
          acc[i][j] = 0.0f;
        }
    }
    if (kt + 1 < nk) {
      store_tiles(buf ^ 1);
      __syncthreads();
    }
  }

#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int64_t r = row_of(i);
    if (r >= M) continue;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int64_t c = col_of(j);
      if (c >= N) continue;
      float* p = C + r + c * ldc;
      if constexpr (CHUNK8) {
        *p = cr[i][j];
      } else {
        if (alpha == -1.0f && beta == 1.0f)
          *p = __fsub_rn(*p, acc[i][j]);
        else if (beta == 0.0f)
          *p = __fmul_rn(alpha, acc[i][j]);
        else
          *p = __fmaf_rn(alpha, acc[i][j], __fmul_rn(beta, *p));
      }
    }
  }
}

// The same product on 64 x 64 tiles (4 x 4 outputs per thread), for
// shapes whose 128 x 128 grid would leave most SMs idle (the narrow FP32
// updates inside a left-looking block: n rows x 128 columns, K = 128).
// Every output's sum runs over K in the same order from 0 and gets the
// same final rounding as in sgemm_update_kernel, so the results are equal.
template <bool VEC>
__global__ void __launch_bounds__(NT)
sgemm_update64_kernel(int64_t M, int64_t N, int64_t K, float alpha,
                      const float* __restrict__ A, int64_t lda,
                      const float* __restrict__ B, int64_t ldb, float beta,
                      float* __restrict__ C, int64_t ldc) {
  constexpr int TB = 64;
  __shared__ __align__(16) float As[2][BK][TB];
  __shared__ __align__(16) float Bs[2][BK][TB];
  const int tid = threadIdx.x;
  const int tx = tid % 16, ty = tid / 16;
  const int64_t m0 = (int64_t)blockIdx.x * TB;
  const int64_t n0 = (int64_t)blockIdx.y * TB;
  // A tile TB x BK: 2 consecutive rows of one column per thread; B tile
  // BK x TB: 2 consecutive k of one column per thread
  const int a_col = tid / 32, a_row = (tid % 32) * 2;
  const int b_col = tid / 4, b_k = (tid % 4) * 2;
  float ra[2], rb[2];
  auto load_tiles = [&](int64_t k0) {
    const int64_t ak = k0 + a_col, ar = m0 + a_row;
    if (VEC && ak < K && ar + 1 < M) {
      const float2 v = *reinterpret_cast<const float2*>(A + ar + ak * lda);
      ra[0] = v.x; ra[1] = v.y;
    } else {
#pragma unroll
      for (int i = 0; i < 2; ++i) ra[i] = (ak < K && ar + i < M) ? A[ar + i + ak * lda] : 0.0f;
    }
    const int64_t bc = n0 + b_col, bk = k0 + b_k;
    if (VEC && bc < N && bk + 1 < K) {
      const float2 v = *reinterpret_cast<const float2*>(B + bk + bc * ldb);
      rb[0] = v.x; rb[1] = v.y;
    } else {
#pragma unroll
      for (int i = 0; i < 2; ++i) rb[i] = (bc < N && bk + i < K) ? B[bk + i + bc * ldb] : 0.0f;
    }
  };
  auto store_tiles = [&](int buf) {
    *reinterpret_cast<float2*>(&As[buf][a_col][a_row]) = make_float2(ra[0], ra[1]);
    Bs[buf][b_k][b_col] = rb[0];
    Bs[buf][b_k + 1][b_col] = rb[1];
  };
  float acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = 0.0f;
  const int64_t nk = (K + BK - 1) / BK;
  load_tiles(0);
  store_tiles(0);
  __syncthreads();
  for (int64_t kt = 0; kt < nk; ++kt) {
    const int buf = (int)(kt & 1);
    if (kt + 1 < nk) load_tiles((kt + 1) * BK);
#pragma unroll
    for (int k = 0; k < BK; ++k) {
      const float4 a4 = *reinterpret_cast<const float4*>(&As[buf][k][tx * 4]);
      const float4 b4 = *reinterpret_cast<const float4*>(&Bs[buf][k][ty * 4]);
      const float a[4] = {a4.x, a4.y, a4.z, a4.w};
      const float b[4] = {b4.x, b4.y, b4.z, b4.w};
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = __fmaf_rn(a[i], b[j], acc[i][j]);
    }
    if (kt + 1 < nk) {
      store_tiles(buf ^ 1);
      __syncthreads();
    }
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int64_t r = m0 + tx * 4 + i;
    if (r >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int64_t c = n0 + ty * 4 + j;
      if (c >= N) continue;
      float* p = C + r + c * ldc;
      if (alpha == -1.0f && beta == 1.0f)
        *p = __fsub_rn(*p, acc[i][j]);
      else if (beta == 0.0f)
        *p = __fmul_rn(alpha, acc[i][j]);
      else
        *p = __fmaf_rn(alpha, acc[i][j], __fmul_rn(beta, *p));
    }
  }
}

// Rank-8-chunked update C -= A * B over up to two independent regions in one
// launch (the rest of an outer block column and of its block row), TM x TM
// outputs per thread on CB x CB tiles (CB = 16 TM: 64 for the wide updates,
// 32 for the small ones, which then get four times as many CTAs): the skinny
// shapes of these updates (K <= 128, one dimension 128 wide) need many small
// tiles to fill the GPU.  Every element's sum runs over K in chunks of 8
// (acc from 0, then subtracted) whatever the tile size.
//
// K <= 128 is small enough to keep the CTA's whole A panel (CB x K) and B
// panel (K x CB) in shared memory: both are requested at once with cp.async
// (A as 16-byte column segments, B transposed by 4-byte copies into rows of
// CB + 4 floats, 4-way bank aliasing at most), the C tile is read while they
// are in flight, and the chunks then run back to back with no barrier.
struct ChunkRegion {
  int64_t M, N, K;
  const float* A; int64_t lda;
  const float* B; int64_t ldb;
  float* C; int64_t ldc;
  int tiles_m, tiles;
};

constexpr int kChunkMaxK = 128;

template <int TM>
constexpr size_t chunk8_smem_bytes() {
  return sizeof(float) * (size_t)kChunkMaxK * (16 * TM + 16 * TM + 4);
}

template <int TM>
__global__ void __launch_bounds__(NT)
sgemm_chunk8_kernel(ChunkRegion r0, ChunkRegion r1) {
  constexpr int CB = 16 * TM;            // tile edge
  constexpr int LB = CB + 4;             // row length of the B panel
  extern __shared__ __align__(16) float smem[];
  float* As = smem;                      // [Kp][CB]: As[k*CB + m]
  float* Bs = smem + kChunkMaxK * CB;    // [Kp][LB]: Bs[k*LB + n]
  const bool second = (int)blockIdx.x >= r0.tiles;
  const ChunkRegion& r = second ? r1 : r0;
  const int t = second ? (int)blockIdx.x - r0.tiles : (int)blockIdx.x;
  const int64_t m0 = (int64_t)(t % r.tiles_m) * CB;
  const int64_t n0 = (int64_t)(t / r.tiles_m) * CB;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int tx = tid % 16, ty = tid / 16;
  const int K = (int)r.K;
  const int Kp = (K + 7) & ~7;           // chunks of 8, zero padded

  // A panel: rows m0.., columns 0..K (column-major in global memory)
  {
    const float* A = r.A + m0;
    const bool vec = ((reinterpret_cast<uintptr_t>(A) & 15) == 0) && (r.lda & 3) == 0 &&
                     m0 + CB <= r.M;
    for (int k = warp; k < Kp; k += NT / 32) {
      float* d = As + k * CB;
      if (vec && k < K) {
        const float* sc = A + (int64_t)k * r.lda;
        for (int m = 4 * lane; m < CB; m += 128) cp_async16(d + m, sc + m);
      } else {
        for (int m = lane; m < CB; m += 32) {
          if (k < K && m0 + m < r.M) cp_async4(d + m, A + m + (int64_t)k * r.lda);
          else d[m] = 0.0f;
        }
      }
    }
  }
  // B panel: rows 0..K, columns n0.. (k contiguous in global memory)
  for (int n = warp; n < CB; n += NT / 32) {
    const bool in = n0 + n < r.N;
    const float* sc = r.B + (n0 + n) * r.ldb;
    for (int k = lane; k < Kp; k += 32) {
      if (in && k < K) cp_async4(Bs + k * LB + n, sc + k);
      else Bs[k * LB + n] = 0.0f;
    }
  }

  float cr[TM][TM], acc[TM][TM];
#pragma unroll
  for (int i = 0; i < TM; ++i)
#pragma unroll
    for (int j = 0; j < TM; ++j) {
      const int64_t row = m0 + tx * TM + i, col = n0 + ty * TM + j;
      cr[i][j] = (row < r.M && col < r.N) ? r.C[row + col * r.ldc] : 0.0f;
      acc[i][j] = 0.0f;
    }
  cp_async_wait_all();
  __syncthreads();

  for (int k0 = 0; k0 < Kp; k0 += 8) {
#pragma unroll
    for (int k = k0; k < k0 + 8; ++k) {
      float a[TM], b[TM];
      if constexpr (TM == 4) {
        const float4 a4 = *reinterpret_cast<const float4*>(As + k * CB + tx * 4);
        const float4 b4 = *reinterpret_cast<const float4*>(Bs + k * LB + ty * 4);
        a[0] = a4.x; a[1] = a4.y; a[2] = a4.z; a[3] = a4.w;
        b[0] = b4.x; b[1] = b4.y; b[2] = b4.z; b[3] = b4.w;
      } else {
        const float2 a2 = *reinterpret_cast<const float2*>(As + k * CB + tx * 2);
        const float2 b2 = *reinterpret_cast<const float2*>(Bs + k * LB + ty * 2);
        a[0] = a2.x; a[1] = a2.y;
        b[0] = b2.x; b[1] = b2.y;
      }
#pragma unroll
      for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int j = 0; j < TM; ++j) acc[i][j] = __fmaf_rn(a[i], b[j], acc[i][j]);
    }
    // one rank-8 chunk done: C -= acc (the reference's K = 8 GEMM)
#pragma unroll
    for (int i = 0; i < TM; ++i)
#pragma unroll
      for (int j = 0; j < TM; ++j) {
        cr[i][j] = __fsub_rn(cr[i][j], acc[i][j]);
        acc[i][j] = 0.0f;
      }
  }
#pragma unroll
  for (int i = 0; i < TM; ++i)
#pragma unroll
    for (int j = 0; j < TM; ++j) {
      const int64_t row = m0 + tx * TM + i, col = n0 + ty * TM + j;
      if (row < r.M && col < r.N) r.C[row + col * r.ldc] = cr[i][j];
    }
}

}  // namespace

lu_status launch_sgemm_chunk8_2(cudaStream_t st, int64_t M0, int64_t N0,
                                int64_t K0, const float* A0, int64_t lda0,
                                const float* B0, int64_t ldb0, float* C0,
                                int64_t ldc0, int64_t M1, int64_t N1, int64_t K1,
                                const float* A1, int64_t lda1, const float* B1,
                                int64_t ldb1, float* C1, int64_t ldc1) {
  ChunkRegion r0{M0, N0, K0, A0, lda0, B0, ldb0, C0, ldc0, 0, 0};
  ChunkRegion r1{M1, N1, K1, A1, lda1, B1, ldb1, C1, ldc1, 0, 0};
  // 64 x 64 tiles unless that leaves fewer than 64 CTAs (then 32 x 32)
  auto count = [&](int cb) {
    int64_t total = 0;
    for (ChunkRegion* r : {&r0, &r1}) {
      r->tiles_m = r->tiles = 0;
      if (r->M > 0 && r->N > 0 && r->K > 0) {
        r->tiles_m = (int)ceil_div(r->M, cb);
        r->tiles = r->tiles_m * (int)ceil_div(r->N, cb);
      }
      total += r->tiles;
    }
    return total;
  };
  int64_t grid = count(64);
  const bool small = grid > 0 && grid < 64;
  if (small) grid = count(32);
  if (grid == 0) return LU_SUCCESS;
  if (grid > INT32_MAX) return LU_ERR_INVALID_ARG;
  if ((r0.tiles > 0 && K0 > kChunkMaxK) || (r1.tiles > 0 && K1 > kChunkMaxK))
    return LU_ERR_INVALID_ARG;
  if (small) {
    constexpr size_t sm = chunk8_smem_bytes<2>();
    LUB_CUDA_TRY(set_smem_limit((const void*)sgemm_chunk8_kernel<2>, sm));
    sgemm_chunk8_kernel<2><<<(unsigned)grid, NT, sm, st>>>(r0, r1);
  } else {
    constexpr size_t sm = chunk8_smem_bytes<4>();
    LUB_CUDA_TRY(set_smem_limit((const void*)sgemm_chunk8_kernel<4>, sm));
    sgemm_chunk8_kernel<4><<<(unsigned)grid, NT, sm, st>>>(r0, r1);
  }
  LUB_LAUNCH_CHECK();
  return LU_SUCCESS;
}

lu_status launch_sgemm_update(cudaStream_t st, int64_t M, int64_t N, int64_t K,
                              float alpha, const float* A, int64_t lda,
                              const float* B, int64_t ldb, float beta, float* C,
                              int64_t ldc, bool chunk8) {
  if (M <= 0 || N <= 0) return LU_SUCCESS;
  if (K <= 0) return LU_SUCCESS;  // nothing to accumulate (beta == 1 callers)
  if (chunk8 && !(alpha == -1.0f && beta == 1.0f)) return LU_ERR_INVALID_ARG;
  const bool vec = (lda % 4 == 0) && (ldb % 4 == 0) &&
                   ((uintptr_t)A % 16 == 0) && ((uintptr_t)B % 16 == 0);
  dim3 grid((unsigned)ceil_div(M, BM), (unsigned)ceil_div(N, BN));
  if (grid.y > 65535) return LU_ERR_INVALID_ARG;
  if (!chunk8 && (int64_t)grid.x * grid.y < 2 * sm_count()) {
    // too few 128 x 128 tiles to fill the GPU: 64 x 64 tiles, same results
    dim3 g64((unsigned)ceil_div(M, 64), (unsigned)ceil_div(N, 64));
    if (g64.y > 65535) return LU_ERR_INVALID_ARG;
    const bool v2 = (lda % 2 == 0) && (ldb % 2 == 0) && ((uintptr_t)A % 8 == 0) &&
                    ((uintptr_t)B % 8 == 0);
    if (v2)
      sgemm_update64_kernel<true><<<g64, NT, 0, st>>>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc);
    else
      sgemm_update64_kernel<false><<<g64, NT, 0, st>>>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc);
    LUB_LAUNCH_CHECK();
    return LU_SUCCESS;
  }
  if (chunk8) {
    if (vec)
      sgemm_update_kernel<true, true><<<grid, NT, 0, st>>>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc);
    else
      sgemm_update_kernel<true, false><<<grid, NT, 0, st>>>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc);
  } else {
    if (vec)
      sgemm_update_kernel<false, true><<<grid, NT, 0, st>>>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc);
    else
      sgemm_update_kernel<false, false><<<grid, NT, 0, st>>>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc);
  }
  LUB_LAUNCH_CHECK();
  return LU_SUCCESS;
}

}  // namespace lub
