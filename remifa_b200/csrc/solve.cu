// Triangular solves with the in-place L\U factors and the FP64 residual of
// iterative refinement.
//
// The reference solves on the host with LAPACK getrs and identity pivots
// (tests/testing_lu_gpu.hxx:1309-1313); its GPU solve is referenced but not
// shipped (tests/testing_lu_gpu.hxx:1353-1359).  Here the solves run on the
// device: the factors stay fp32 (4 bytes per element read per solve, the
// bandwidth that bounds a triangular solve), the right-hand sides and all
// arithmetic are fp64, so the solve adds no fp32 rounding on top of the
// factorization error -- what iterative refinement in fp64 needs.
//
// op(T) X = B, T = L (unit lower) or U (upper), op = identity or transpose,
// runs as ONE launch per triangle (trsv_kernel): a CTA per (row block of 64
// rows, group of up to 8 right-hand sides).  CTAs draw tickets in solve
// order (an atomic counter), so a CTA only ever waits for CTAs that are
// already running: no deadlock whatever the residency.  Row block t
// streams the 64 x 64 tiles op(T)[t, q] of the blocks solved before it
// through a cp.async ring in shared memory, consuming each as soon as that
// block's solution is published (a per-group counter of finished blocks,
// release / acquire at GPU scope) and accumulating per lane in fp64; tiles
// are fetched ahead of the solve front, so the factor streams at memory
// speed while the front advances.  The diagonal block is inverted (fp64
// substitution, off the critical path while the CTA waits) and applied as
// a 64 x 64 product, so the step that hands the solution from block to
// block is one tile product, one shuffle reduction and one small product.
// Every wait is bounded (a few seconds of %globaltimer); on expiry the CTA
// raises the abort word, every later CTA stops waiting, and the rows of the
// CTAs that gave up are written as NaN, so a failed solve never looks like
// a result.
#include "common.cuh"
#include "kernels.cuh"
#include "solve.cuh"

namespace lub {
namespace {

constexpr int kT = 256;    // threads per CTA of the residual kernels

namespace trsv {

constexpr int BS = 64;                 // rows of a row block = columns of a tile
constexpr int kThreads = 256;          // 8 warps; warp w owns rows 8w .. 8w+7
constexpr int S = 4;                   // ring stages
constexpr int kSyncHeader = 4;         // ticket, abort, timeouts, spare
constexpr unsigned long long kWaitNs = 4000000000ull;  // bound of one wait

__host__ __device__ constexpr size_t smem_bytes(int nr) {
  return (size_t)S * BS * BS * 4          // fp32 tiles
         + (size_t)S * nr * BS * 8        // fp64 solution blocks of the tiles
         + (size_t)BS * BS * 8            // inverse of the diagonal block
         + (size_t)nr * BS * 8            // right-hand side / y
         + (size_t)4 * nr * BS * 8        // partial sums of the final product
         + 64;                            // control words
}

struct Args {
  const float* lu;
  int64_t ld;
  double* X;
  int64_t ldx;
  int64_t n;
  int64_t nrhs;
  int nblk;
  int ngroups;
  int forward;   // op(T) lower: L or U^T
  int unit;      // unit diagonal: L or L^T
  int xvec;      // X 16-byte aligned with even ldx: solution blocks by cp.async
  unsigned* sync;
};

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(unsigned* p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// cp.async with zero fill: copies src_bytes (0 .. size) and zeroes the rest.
__device__ __forceinline__ void cp16z(void* dst, const void* src, int src_bytes) {
  const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(dst));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(src),
               "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp4z(void* dst, const void* src, int src_bytes) {
  const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(dst));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(d), "l"(src),
               "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

__device__ __forceinline__ int imin64(int64_t a, int b) { return a < b ? (int)a : b; }

// Shared-memory layout of a 64 x 64 tile of op(T) (rows r, columns k).
// Not transposed: column k of op(T) is column k0+k of the factor, contiguous
// in r; stored by 16-byte chunks (4 rows) with chunk index q ^ (k & 7), so
// that 8 lanes reading chunk q of 8 consecutive columns hit 8 different
// bank groups.  Transposed: row r of op(T) is contiguous in k; stored
// row-major, lanes read consecutive k.
template <bool TRANS>
__device__ __forceinline__ int tile_index(int r, int k) {
  return TRANS ? r * BS + k : k * BS + 4 * ((r >> 2) ^ (k & 7)) + (r & 3);
}

// Issue the copy of tile op(T)[rows r0.., cols k0..] (rw x kw valid, the
// rest zero) into dst.
template <bool TRANS, bool V16>
__device__ __forceinline__ void load_tile(float* dst, const Args& a, int64_t r0, int rw,
                                          int64_t k0, int kw) {
  const int tid = threadIdx.x;
  if (V16) {
#pragma unroll
    for (int m = 0; m < BS * BS / 4 / kThreads; ++m) {
      const int c = tid + m * kThreads;
      const int outer = c >> 4, q = c & 15;   // outer: k (or r), q: chunk of 4
      int64_t mcol, mrow;                     // memory column, first memory row
      int valid;                              // valid elements of the chunk
      if (!TRANS) {
        mcol = k0 + outer; mrow = r0 + 4 * q;
        valid = outer < kw ? min(4, max(0, rw - 4 * q)) : 0;
      } else {
        mcol = r0 + outer; mrow = k0 + 4 * q;
        valid = outer < rw ? min(4, max(0, kw - 4 * q)) : 0;
      }
      const float* src = valid ? a.lu + mrow + mcol * a.ld : a.lu;
      float* d = TRANS ? dst + outer * BS + 4 * q : dst + outer * BS + 4 * (q ^ (outer & 7));
      cp16z(d, src, valid * 4);
    }
  } else {
#pragma unroll 4
    for (int m = 0; m < BS * BS / kThreads; ++m) {
      const int e = tid + m * kThreads;
      const int outer = e >> 6, inner = e & 63;
      if (!TRANS) {
        const bool ok = outer < kw && inner < rw;
        cp4z(dst + tile_index<false>(inner, outer),
             ok ? a.lu + (r0 + inner) + (k0 + outer) * a.ld : a.lu, ok ? 4 : 0);
      } else {
        const bool ok = outer < rw && inner < kw;
        cp4z(dst + tile_index<true>(outer, inner),
             ok ? a.lu + (k0 + inner) + (r0 + outer) * a.ld : a.lu, ok ? 4 : 0);
      }
    }
  }
}

// Issue the copy of the diagonal block as plain fp32: memory column c,
// memory row r of the block at c * 64 + r (the rest zero).
template <bool V16>
__device__ __forceinline__ void load_diag(float* dst, const Args& a, int64_t r0, int rw) {
  const int tid = threadIdx.x;
  if (V16) {
#pragma unroll
    for (int m = 0; m < BS * BS / 4 / kThreads; ++m) {
      const int c = tid + m * kThreads;
      const int outer = c >> 4, q = c & 15;
      const int valid = outer < rw ? min(4, max(0, rw - 4 * q)) : 0;
      const float* src = valid ? a.lu + (r0 + 4 * q) + (r0 + outer) * a.ld : a.lu;
      cp16z(dst + outer * BS + 4 * q, src, valid * 4);
    }
  } else {
#pragma unroll 4
    for (int m = 0; m < BS * BS / kThreads; ++m) {
      const int e = tid + m * kThreads;
      const int outer = e >> 6, inner = e & 63;
      const bool ok = outer < rw && inner < rw;
      cp4z(dst + outer * BS + inner, ok ? a.lu + (r0 + inner) + (r0 + outer) * a.ld : a.lu,
           ok ? 4 : 0);
    }
  }
}

// Solution block of a tile: rows k0 .. k0+kw of the group's columns, the
// rest zero.  Async form: 16-byte copies through L2 (the block was written
// by another SM; L1 is bypassed).  Sync form: plain L2 loads.
template <int NR>
__device__ __forceinline__ void load_x_async(double* dst, const Args& a, int64_t k0, int kw,
                                             int64_t c0, int nc) {
  for (int e = threadIdx.x; e < NR * BS / 2; e += kThreads) {
    const int c = e / (BS / 2), k = 2 * (e % (BS / 2));
    const int valid = c < nc ? min(2, max(0, kw - k)) : 0;
    const double* src = valid ? a.X + (k0 + k) + (c0 + c) * a.ldx : a.X;
    cp16z(dst + c * BS + k, src, valid * 8);
  }
}
template <int NR>
__device__ __forceinline__ void load_x_sync(double* dst, const Args& a, int64_t k0, int kw,
                                            int64_t c0, int nc) {
  for (int e = threadIdx.x; e < NR * BS; e += kThreads) {
    const int c = e / BS, k = e % BS;
    dst[e] = (c < nc && k < kw) ? __ldcg(a.X + (k0 + k) + (c0 + c) * a.ldx) : 0.0;
  }
}

template <bool TRANS, int NR, bool V16>
__global__ void __launch_bounds__(kThreads, NR >= 8 ? 1 : 2)
trsv_kernel(Args a) {
  extern __shared__ __align__(16) unsigned char smem[];
  float* Tr = reinterpret_cast<float*>(smem);
  double* Xr = reinterpret_cast<double*>(smem + (size_t)S * BS * BS * 4);
  double* Dinv = Xr + S * NR * BS;
  double* ybuf = Dinv + BS * BS;
  double* red = ybuf + NR * BS;
  int* ctrl = reinterpret_cast<int*>(red + 4 * NR * BS);  // ticket, avail[2], abort

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  unsigned* abort_word = a.sync + 1;
  if (tid == 0) {
    const unsigned tk = atomicAdd(a.sync, 1u);
    ctrl[0] = (int)tk;
    ctrl[1] = (int)ld_acquire(a.sync + kSyncHeader + tk % (unsigned)a.ngroups);
    ctrl[3] = 0;
  }
  __syncthreads();
  const int ticket = ctrl[0];
  const int t = ticket / a.ngroups, g = ticket - t * a.ngroups;
  const bool fwd = a.forward != 0;
  const int64_t r0 = (int64_t)(fwd ? t : a.nblk - 1 - t) * BS;
  const int rw = imin64(a.n - r0, BS);
  const int64_t c0 = (int64_t)g * NR;
  const int nc = imin64(a.nrhs - c0, NR);
  unsigned* done = a.sync + kSyncHeader + g;

  // column offset / width of the tile at solve position q
  auto tile_k0 = [&](int q) -> int64_t { return (int64_t)(fwd ? q : a.nblk - 1 - q) * BS; };
  auto tile_kw = [&](int q) -> int { return imin64(a.n - tile_k0(q), BS); };

  // right-hand side rows of this block
  for (int e = tid; e < NR * BS; e += kThreads) {
    const int c = e / BS, r = e % BS;
    ybuf[e] = (c < nc && r < rw) ? a.X[(r0 + r) + (c0 + c) * a.ldx] : 0.0;
  }
  // diagonal block (fp32, in the inverse's space), then the ring prologue
  float* Dsrc = reinterpret_cast<float*>(Dinv);
  load_diag<V16>(Dsrc, a, r0, rw);
  cp_commit();
  int avail = ctrl[1];
  unsigned xbits = 0;
  auto issue = [&](int q) {
    if (q < t) {
      const int st = q % S;
      const int64_t k0 = tile_k0(q);
      const int kw = tile_kw(q);
      load_tile<TRANS, V16>(Tr + st * BS * BS, a, r0, rw, k0, kw);
      if (a.xvec && q < avail) {
        load_x_async<NR>(Xr + st * NR * BS, a, k0, kw, c0, nc);
        xbits |= 1u << st;
      } else {
        xbits &= ~(1u << st);
      }
    }
    cp_commit();
  };
#pragma unroll 1
  for (int q = 0; q < S - 1; ++q) issue(q);

  // ---- inverse of the diagonal block: fp64 substitution, column j by the
  // four lanes 4j .. 4j+3, lane part p holding rows 4s + p ----
  cp_wait<S - 1>();
  __syncthreads();
  if (rw < BS && tid >= rw && tid < BS) Dsrc[tid * BS + tid] = 1.0f;  // identity padding
  __syncthreads();
  {
    const int j = tid >> 2, p = tid & 3;
    // element (r, k) of op(T): memory row r, column k (or the transpose)
    auto D = [&](int r, int k) -> double {
      return (double)(TRANS ? Dsrc[r * BS + k] : Dsrc[k * BS + r]);
    };
    double z[16];
#pragma unroll
    for (int s = 0; s < 16; ++s) z[s] = (4 * s + p == j) ? 1.0 : 0.0;
    const bool unit = a.unit != 0;
    if (fwd) {
#pragma unroll
      for (int k = 0; k < BS; ++k) {
        const bool live = k >= j;
        if (live && !unit && p == (k & 3)) z[k >> 2] = z[k >> 2] / D(k, k);
        const double zk = __shfl_sync(0xffffffffu, z[k >> 2], (lane & ~3) | (k & 3));
        if (live) {
#pragma unroll
          for (int s = 0; s < 16; ++s)
            if (4 * s + p > k) z[s] = fma(-D(4 * s + p, k), zk, z[s]);
        }
      }
    } else {
#pragma unroll
      for (int k = BS - 1; k >= 0; --k) {
        const bool live = k <= j;
        if (live && !unit && p == (k & 3)) z[k >> 2] = z[k >> 2] / D(k, k);
        const double zk = __shfl_sync(0xffffffffu, z[k >> 2], (lane & ~3) | (k & 3));
        if (live) {
#pragma unroll
          for (int s = 0; s < 16; ++s)
            if (4 * s + p < k) z[s] = fma(-D(4 * s + p, k), zk, z[s]);
        }
      }
    }
    __syncthreads();  // every read of the fp32 block precedes the overwrite
#pragma unroll
    for (int s = 0; s < 16; ++s) Dinv[j * BS + 4 * s + p] = z[s];
  }

  // ---- stream the tiles of the blocks solved before this one ----
  double acc[8][NR];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int c = 0; c < NR; ++c) acc[i][c] = 0.0;
  int refresh = 0;
  bool aborted = false;
#pragma unroll 1
  for (int q = 0; q < t; ++q) {
    if (q >= avail) {
      // wait until solve position q is published (thread 0 polls, bounded)
      if (tid == 0) {
        unsigned v = ld_acquire(done);
        if ((int)v <= q) {
          const unsigned long long t0 = global_ns();
          for (;;) {
            v = ld_acquire(done);
            if ((int)v > q) break;
            if (*(volatile unsigned*)abort_word) { ctrl[3] = 1; break; }
            if (global_ns() - t0 > kWaitNs) {
              atomicExch(abort_word, 1u);
              atomicAdd(a.sync + 2, 1u);
              ctrl[3] = 1;
              break;
            }
          }
        }
        ctrl[1 + (refresh & 1)] = (int)v;
      }
      __syncthreads();
      avail = ctrl[1 + (refresh & 1)];
      ++refresh;
      if (ctrl[3]) { aborted = true; break; }
    }
    const int st = q % S;
    cp_wait<S - 2>();
    if (!((xbits >> st) & 1u))
      load_x_sync<NR>(Xr + st * NR * BS, a, tile_k0(q), tile_kw(q), c0, nc);
    __syncthreads();
    issue(q + S - 1);
    const float* Ts = Tr + st * BS * BS;
    const double* xs = Xr + st * NR * BS;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int k = lane + 32 * h;
      double xv[NR];
#pragma unroll
      for (int c = 0; c < NR; ++c) xv[c] = xs[c * BS + k];
      float tv[8];
      if (!TRANS) {
        const float4 u0 = *reinterpret_cast<const float4*>(Ts + tile_index<false>(8 * warp, k));
        const float4 u1 = *reinterpret_cast<const float4*>(Ts + tile_index<false>(8 * warp + 4, k));
        tv[0] = u0.x; tv[1] = u0.y; tv[2] = u0.z; tv[3] = u0.w;
        tv[4] = u1.x; tv[5] = u1.y; tv[6] = u1.z; tv[7] = u1.w;
      } else {
#pragma unroll
        for (int i = 0; i < 8; ++i) tv[i] = Ts[tile_index<true>(8 * warp + i, k)];
      }
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int c = 0; c < NR; ++c) acc[i][c] = fma((double)tv[i], xv[c], acc[i][c]);
    }
  }
  cp_wait<0>();
  if (aborted) {
    for (int e = tid; e < NR * BS; e += kThreads) {
      const int c = e / BS, r = e % BS;
      if (c < nc && r < rw)
        a.X[(r0 + r) + (c0 + c) * a.ldx] = __longlong_as_double(0x7ff8000000000000ll);
    }
    return;
  }

  // ---- y = b - sum: each row reduced over the 32 lanes (three halving
  // exchanges, then two full steps); lane 4i ends with row 8 warp + i ----
#pragma unroll
  for (int c = 0; c < NR; ++c) {
    double v[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = acc[i][c];
    const bool b4 = lane & 16, b3 = lane & 8, b2 = lane & 4;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const double send = b4 ? v[i] : v[i + 4];
      const double keep = b4 ? v[i + 4] : v[i];
      v[i] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
    }
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const double send = b3 ? v[i] : v[i + 2];
      const double keep = b3 ? v[i + 2] : v[i];
      v[i] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
    }
    {
      const double send = b2 ? v[0] : v[1];
      const double keep = b2 ? v[1] : v[0];
      v[0] = keep + __shfl_xor_sync(0xffffffffu, send, 4);
    }
    v[0] += __shfl_xor_sync(0xffffffffu, v[0], 2);
    v[0] += __shfl_xor_sync(0xffffffffu, v[0], 1);
    if ((lane & 3) == 0) ybuf[c * BS + 8 * warp + (lane >> 2)] -= v[0];
  }
  __syncthreads();

  // ---- x = Dinv y: row r = tid & 63, quarter p of the columns ----
  {
    const int r = tid & 63, p = tid >> 6;
    double part[NR];
#pragma unroll
    for (int c = 0; c < NR; ++c) part[c] = 0.0;
#pragma unroll
    for (int jj = 0; jj < 16; ++jj) {
      const int j = 16 * p + jj;
      const double d = Dinv[j * BS + r];
#pragma unroll
      for (int c = 0; c < NR; ++c) part[c] = fma(d, ybuf[c * BS + j], part[c]);
    }
#pragma unroll
    for (int c = 0; c < NR; ++c) red[(p * NR + c) * BS + r] = part[c];
  }
  __syncthreads();
  for (int e = tid; e < NR * BS; e += kThreads) {
    const int c = e / BS, r = e % BS;
    const double x = ((red[(0 * NR + c) * BS + r] + red[(1 * NR + c) * BS + r]) +
                      red[(2 * NR + c) * BS + r]) + red[(3 * NR + c) * BS + r];
    if (c < nc && r < rw) a.X[(r0 + r) + (c0 + c) * a.ldx] = x;
  }
  __syncthreads();
  if (tid == 0) st_release(done, (unsigned)(t + 1));
}

int group_width(int64_t nrhs) { return nrhs >= 8 ? 8 : nrhs >= 4 ? 4 : nrhs >= 2 ? 2 : 1; }

template <bool TRANS, int NR, bool V16>
lu_status launch_one(cudaStream_t st, const Args& a) {
  const size_t smem = smem_bytes(NR);
  auto fn = trsv_kernel<TRANS, NR, V16>;
  LUB_CUDA_TRY(set_smem_limit((const void*)fn, smem));
  fn<<<(unsigned)((int64_t)a.nblk * a.ngroups), kThreads, smem, st>>>(a);
  LUB_LAUNCH_CHECK();
  return LU_SUCCESS;
}

template <bool TRANS, bool V16>
lu_status launch_nr(cudaStream_t st, const Args& a, int nr) {
  switch (nr) {
    case 8: return launch_one<TRANS, 8, V16>(st, a);
    case 4: return launch_one<TRANS, 4, V16>(st, a);
    case 2: return launch_one<TRANS, 2, V16>(st, a);
    default: return launch_one<TRANS, 1, V16>(st, a);
  }
}

}  // namespace trsv

// ---- residual r = b - A x (fp32 A, fp64 b, x, r) -------------------------
// Column chunks of kRC columns give partial dot products P[chunk][row]; a
// second pass adds them in chunk order, so the result does not depend on
// scheduling.
constexpr int kRC = 256;

__global__ void __launch_bounds__(kT)
residual_partial_kernel(int64_t n, const float* __restrict__ A, int64_t lda,
                        const double* __restrict__ x, double* __restrict__ P) {
  __shared__ double xs[kRC];
  const int64_t c0 = (int64_t)blockIdx.y * kRC;
  const int cn = (int)((n - c0) < kRC ? (n - c0) : kRC);
  for (int k = threadIdx.x; k < cn; k += kT) xs[k] = x[c0 + k];
  __syncthreads();
  const int64_t i = (int64_t)blockIdx.x * kT + threadIdx.x;
  if (i >= n) return;
  const float* col = A + i + c0 * lda;
  double acc = 0.0;
#pragma unroll 8
  for (int k = 0; k < cn; ++k) acc = fma((double)col[k * lda], xs[k], acc);
  P[(int64_t)blockIdx.y * n + i] = acc;
}

// r = b - sum_chunks P; also the row sums |A| once (rowsum != null) and the
// maxima needed for the backward error (atomicMax on non-negative doubles
// through their bit patterns).
__global__ void __launch_bounds__(kT)
residual_final_kernel(int64_t n, int nchunks, const double* __restrict__ P,
                      const double* __restrict__ b, const double* __restrict__ x,
                      double* __restrict__ r, unsigned long long* __restrict__ maxes) {
  const int64_t i = (int64_t)blockIdx.x * kT + threadIdx.x;
  double ri = 0.0, xi = 0.0, bi = 0.0;
  if (i < n) {
    double s = 0.0;
    for (int c = 0; c < nchunks; ++c) s += P[(int64_t)c * n + i];
    bi = b[i];
    ri = bi - s;
    r[i] = ri;
    xi = x[i];
  }
  // maxes[0] = max |r|, [1] = max |x|, [2] = max |b|
  double v[3] = {fabs(ri), fabs(xi), fabs(bi)};
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    double m = v[q];
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(&maxes[q], (unsigned long long)__double_as_longlong(m));
  }
}

// max_i sum_j |a_ij| (the infinity norm), same chunked scheme.
__global__ void __launch_bounds__(kT)
rowsum_partial_kernel(int64_t n, const float* __restrict__ A, int64_t lda,
                      double* __restrict__ P) {
  const int64_t c0 = (int64_t)blockIdx.y * kRC;
  const int cn = (int)((n - c0) < kRC ? (n - c0) : kRC);
  const int64_t i = (int64_t)blockIdx.x * kT + threadIdx.x;
  if (i >= n) return;
  const float* col = A + i + c0 * lda;
  double acc = 0.0;
  for (int k = 0; k < cn; ++k) acc += fabs((double)col[k * lda]);
  P[(int64_t)blockIdx.y * n + i] = acc;
}

__global__ void __launch_bounds__(kT)
rowsum_final_kernel(int64_t n, int nchunks, const double* __restrict__ P,
                    unsigned long long* __restrict__ out) {
  const int64_t i = (int64_t)blockIdx.x * kT + threadIdx.x;
  double s = 0.0;
  if (i < n)
    for (int c = 0; c < nchunks; ++c) s += P[(int64_t)c * n + i];
  for (int o = 16; o > 0; o >>= 1) s = fmax(s, __shfl_xor_sync(0xffffffffu, s, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(s));
}

__global__ void axpy_kernel(int64_t n, const double* __restrict__ d,
                            double* __restrict__ x) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] += d[i];
}

}  // namespace

size_t trsm_sync_bytes(int64_t nrhs) {
  const int64_t groups = ceil_div(nrhs < 1 ? 1 : nrhs, trsv::group_width(nrhs));
  return align_up((size_t)(trsv::kSyncHeader + groups) * 4, 256);
}

lu_status launch_trsm(cudaStream_t st, int64_t n, const float* lu, int64_t ld,
                      double* X, int64_t ldx, int64_t nrhs, bool upper,
                      bool trans, void* sync) {
  if (n <= 0 || nrhs <= 0) return LU_SUCCESS;
  if (!sync) return LU_ERR_INVALID_ARG;
  const int nr = trsv::group_width(nrhs);
  trsv::Args a;
  a.lu = lu;
  a.ld = ld;
  a.X = X;
  a.ldx = ldx;
  a.n = n;
  a.nrhs = nrhs;
  if (ceil_div(n, trsv::BS) * ceil_div(nrhs, nr) > 0x7fffffffll) return LU_ERR_INVALID_ARG;
  a.nblk = (int)ceil_div(n, trsv::BS);
  a.ngroups = (int)ceil_div(nrhs, nr);
  // op(T) is lower (forward substitution) for L and for U^T
  a.forward = upper == trans;
  a.unit = !upper;
  a.xvec = ((reinterpret_cast<uintptr_t>(X) & 15) == 0) && (ldx % 2 == 0);
  a.sync = static_cast<unsigned*>(sync);
  LUB_CUDA_TRY(cudaMemsetAsync(sync, 0, (size_t)(trsv::kSyncHeader + a.ngroups) * 4, st));
  const bool v16 = ((reinterpret_cast<uintptr_t>(lu) & 15) == 0) && (ld % 4 == 0);
  if (trans)
    return v16 ? trsv::launch_nr<true, true>(st, a, nr) : trsv::launch_nr<true, false>(st, a, nr);
  return v16 ? trsv::launch_nr<false, true>(st, a, nr) : trsv::launch_nr<false, false>(st, a, nr);
}

lu_status launch_lu_solve(cudaStream_t st, int64_t n, const float* lu, int64_t ld,
                          double* X, int64_t ldx, int64_t nrhs, bool trans, void* sync) {
  if (!trans) {  // L U x = b: L y = b, then U x = y
    LUB_TRY(launch_trsm(st, n, lu, ld, X, ldx, nrhs, false, false, sync));
    return launch_trsm(st, n, lu, ld, X, ldx, nrhs, true, false, sync);
  }
  // (L U)^T x = U^T L^T x = b: U^T y = b, then L^T x = y
  LUB_TRY(launch_trsm(st, n, lu, ld, X, ldx, nrhs, true, true, sync));
  return launch_trsm(st, n, lu, ld, X, ldx, nrhs, false, true, sync);
}

size_t residual_ws_bytes(int64_t n) {
  return align_up((size_t)ceil_div(n, kRC) * n * sizeof(double), 256) + 256;
}

lu_status launch_residual(cudaStream_t st, int64_t n, const float* A,
                          int64_t lda, const double* b, const double* x,
                          double* r, void* ws, unsigned long long* maxes) {
  const int nch = (int)ceil_div(n, kRC);
  double* P = static_cast<double*>(ws);
  LUB_CUDA_TRY(cudaMemsetAsync(maxes, 0, 3 * sizeof(unsigned long long), st));
  dim3 g((unsigned)ceil_div(n, kT), (unsigned)nch);
  residual_partial_kernel<<<g, kT, 0, st>>>(n, A, lda, x, P);
  LUB_LAUNCH_CHECK();
  residual_final_kernel<<<(unsigned)ceil_div(n, kT), kT, 0, st>>>(n, nch, P, b, x, r, maxes);
  LUB_LAUNCH_CHECK();
  return LU_SUCCESS;
}

lu_status launch_norm_inf(cudaStream_t st, int64_t n, const float* A,
                          int64_t lda, void* ws, unsigned long long* out) {
  const int nch = (int)ceil_div(n, kRC);
  double* P = static_cast<double*>(ws);
  LUB_CUDA_TRY(cudaMemsetAsync(out, 0, sizeof(unsigned long long), st));
  dim3 g((unsigned)ceil_div(n, kT), (unsigned)nch);
  rowsum_partial_kernel<<<g, kT, 0, st>>>(n, A, lda, P);
  LUB_LAUNCH_CHECK();
  rowsum_final_kernel<<<(unsigned)ceil_div(n, kT), kT, 0, st>>>(n, nch, P, out);
  LUB_LAUNCH_CHECK();
  return LU_SUCCESS;
}

lu_status launch_axpy(cudaStream_t st, int64_t n, const double* d, double* x) {
  axpy_kernel<<<(unsigned)ceil_div(n, 256), 256, 0, st>>>(n, d, x);
  LUB_LAUNCH_CHECK();
  return LU_SUCCESS;
}

}  // namespace lub
