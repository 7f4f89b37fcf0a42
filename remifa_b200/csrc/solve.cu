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
// runs as one launch per triangle (trsv_kernel) after a copy kernel that
// moves B aside and marks every entry of X pending (a signalling-NaN
// pattern no arithmetic produces).  A CTA per (row block of 64 rows, group
// of up to 8 right-hand sides); CTAs draw tickets in solve order (an atomic
// counter), so a CTA only ever waits for CTAs already running: no deadlock
// whatever the residency.  Each warp of a CTA owns 8 rows of the block and
// streams its share of the tiles op(T)[t, q] of the blocks solved earlier
// through its own cp.async ring, reading the solution entries it needs
// straight from X (relaxed loads at GPU scope, re-read while pending; the
// solution IS the flag, so publishing a block costs one store, no fence and
// no counter).  The diagonal block is inverted in fp64 and the last tile is
// folded into W = Dinv op(T)[t, t-1] while the CTA waits, so the hand-over
// from block t-1 to block t is, per warp and without a CTA barrier:
// x_t = Dinv (b - sum_{q<t-1} op(T)[t,q] x_q) - W x_{t-1}, i.e. 16 fma per
// lane and one shuffle reduction after x_{t-1} lands.
#include "common.cuh"
#include "kernels.cuh"
#include "solve.cuh"

namespace lub {
namespace {

constexpr int kT = 256;    // threads per CTA of the residual kernels

namespace trsv {

constexpr int BS = 64;                 // rows of a row block = columns of a tile
constexpr int kThreads = 256;          // 8 warps
constexpr unsigned long long kWaitNs = 4000000000ull;  // bound of one wait

struct Args {
  const float* lu;
  int64_t ld;
  double* X;        // solutions, written in place
  int64_t ldx;
  const double* B;  // right-hand sides (n x nrhs, ld n) of the warp kernel
  int64_t n;
  int64_t nrhs;
  int nblk;
  int ngroups;
  int forward;      // op(T) lower: L or U^T
  int unit;         // unit diagonal: L or L^T
  int xvec;         // X 16-byte aligned with even ldx (group kernel: cp.async)
  unsigned* sync;
  unsigned long long wait_ns;  // bound of one wait (kWaitNs)
  int withhold;     // self-test of the give-up path only: the row block solved
                    // first (ticket 0) does not publish its solution, -1: none
};

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

// Shared layout of a full 64 x 64 tile of op(T) (rows r, columns k).  Not
// transposed: column k contiguous in r, by 16-byte chunks with chunk index
// (r/4) ^ (k & 7) (8 lanes reading one chunk of 8 consecutive columns hit 8
// bank groups).  Transposed: row-major.
template <bool TRANS>
__device__ __forceinline__ int tile_index(int r, int k) {
  return TRANS ? r * BS + k : k * BS + 4 * ((r >> 2) ^ (k & 7)) + (r & 3);
}

// Copy of the full tile op(T)[rows r0.., cols k0..] (rw x kw valid, the rest
// zero), all threads of the CTA.
template <bool TRANS, bool V16>
__device__ __forceinline__ void load_tile(float* dst, const Args& a, int64_t r0, int rw,
                                          int64_t k0, int kw) {
  const int tid = threadIdx.x;
  if (V16) {
#pragma unroll
    for (int m = 0; m < BS * BS / 4 / kThreads; ++m) {
      const int c = tid + m * kThreads;
      const int outer = c >> 4, q = c & 15;
      int64_t mcol, mrow;
      int valid;
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

// Copy of the diagonal block as plain fp32: memory column c, memory row r of
// the block at c * 64 + r (the rest zero), all threads of the CTA.
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

// Inverse of the diagonal block of op(T) (fp32 in Dsrc as load_diag left it)
// by fp64 substitution with the reciprocals of the diagonal: column j by
// lanes 4j .. 4j+3, part p holding rows 4s + p.  Written row-major into
// Dinv[r * 64 + j] (the same space as Dsrc; a barrier separates the reads
// from the writes).  Rows and columns past rw are the identity.  All threads.
template <bool TRANS>
__device__ __forceinline__ void invert_diag(const float* Dsrc, double* Dinv, double* rdiag,
                                            int rw, bool fwd, bool unit) {
  const int tid = threadIdx.x, lane = tid & 31;
  auto D = [&](int r, int k) -> double {
    return (double)(TRANS ? Dsrc[r * BS + k] : Dsrc[k * BS + r]);
  };
  if (tid < BS) rdiag[tid] = (unit || tid >= rw) ? 1.0 : 1.0 / D(tid, tid);
  __syncthreads();
  const int j = tid >> 2, p = tid & 3;
  double z[16];
#pragma unroll
  for (int s = 0; s < 16; ++s) z[s] = (4 * s + p == j) ? 1.0 : 0.0;
  if (fwd) {
#pragma unroll
    for (int k = 0; k < BS; ++k) {
      const bool live = k >= j;
      if (live && p == (k & 3)) z[k >> 2] *= rdiag[k];
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
      if (live && p == (k & 3)) z[k >> 2] *= rdiag[k];
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
  for (int s = 0; s < 16; ++s) Dinv[(4 * s + p) * BS + j] = z[s];
  __syncthreads();
}

// Sum over the 32 lanes of each of 8 per-lane partial rows: three halving
// exchanges, then two full steps.  Lanes 4i .. 4i+3 end with row i.
__device__ __forceinline__ double row_reduce(double (&v)[8], int lane) {
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
  double s;
  {
    const double send = b2 ? v[0] : v[1];
    const double keep = b2 ? v[1] : v[0];
    s = keep + __shfl_xor_sync(0xffffffffu, send, 4);
  }
  s += __shfl_xor_sync(0xffffffffu, s, 2);
  s += __shfl_xor_sync(0xffffffffu, s, 1);
  return s;
}

// ======================================================================
// Warp kernel (groups of 1 or 2 right-hand sides).  X is marked pending by
// trsv_prepare_kernel; a solution entry is published by one store and read
// by relaxed loads at GPU scope, re-read while pending -- the solution is
// its own flag.
// ======================================================================

constexpr int S = 3;                   // stages of each warp's tile ring
constexpr int kWarpTile = 8 * BS;      // floats of a warp's share of a tile
// Marks a solution entry not yet published: a signalling-NaN payload that no
// arithmetic produces (published NaNs are stored as the canonical quiet NaN).
constexpr unsigned long long kPending = 0x7ff4dead5e1f5e1full;
constexpr unsigned long long kQuietNaN = 0x7ff8000000000000ull;

__host__ __device__ constexpr size_t warp_smem_bytes(int nr) {
  return (size_t)S * 8 * kWarpTile * 4    // per-warp tile rings (fp32)
         + (size_t)BS * BS * 8            // inverse of the diagonal block (fp64)
         + (size_t)BS * BS * 4            // tile of the previous block (fp32)
         + (size_t)8 * nr * BS * 8        // per-warp partial sums
         + (size_t)BS * 8                 // reciprocals of the diagonal
         + 64;                            // control words
}

__device__ __forceinline__ double ld_poll(const double* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return __longlong_as_double((long long)v);
}
__device__ __forceinline__ void st_publish(double* p, double x) {
  unsigned long long v = (unsigned long long)__double_as_longlong(x);
  if ((v & 0x7ff0000000000000ull) == 0x7ff0000000000000ull && (v & 0xfffffffffffffull))
    v = kQuietNaN;
  asm volatile("st.relaxed.gpu.global.b64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ bool pending(double x) {
  return (unsigned long long)__double_as_longlong(x) == kPending;
}

// A warp's share of a tile.  Transposed (row share): rows 8w .. 8w+7 of the
// block, row-major [i][k] (each row of op(T) is 256 contiguous bytes of one
// factor column).  Not transposed (column share): columns 8w .. 8w+7 of the
// tile, [j][r] (each column 256 contiguous bytes).  Copied by the warp's
// own lanes.
template <bool TRANS, bool V16>
__device__ __forceinline__ void load_warp_tile(float* dst, const Args& a, int64_t r0, int rw,
                                               int64_t k0, int kw, int w, int lane) {
  const int b = 8 * w;
  if (V16) {
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      const int c = lane + 32 * m;
      const int o = c >> 4, q = c & 15;
      int valid;
      const float* src;
      if (!TRANS) {
        valid = b + o < kw ? min(4, max(0, rw - 4 * q)) : 0;
        src = valid ? a.lu + (r0 + 4 * q) + (k0 + b + o) * a.ld : a.lu;
      } else {
        valid = b + o < rw ? min(4, max(0, kw - 4 * q)) : 0;
        src = valid ? a.lu + (k0 + 4 * q) + (r0 + b + o) * a.ld : a.lu;
      }
      cp16z(dst + o * BS + 4 * q, src, valid * 4);
    }
  } else {
#pragma unroll 4
    for (int m = 0; m < 16; ++m) {
      const int e = lane + 32 * m;
      const int o = e >> 6, i = e & 63;
      bool ok;
      const float* src;
      if (!TRANS) {
        ok = b + o < kw && i < rw;
        src = ok ? a.lu + (r0 + i) + (k0 + b + o) * a.ld : a.lu;
      } else {
        ok = b + o < rw && i < kw;
        src = ok ? a.lu + (k0 + i) + (r0 + b + o) * a.ld : a.lu;
      }
      cp4z(dst + o * BS + i, src, ok ? 4 : 0);
    }
  }
}

// Solution entries of tile columns kb + h*ks (h < NX) of the group's
// columns (0 outside the matrix), as loaded -- possibly still pending.
template <int NX, int NR>
__device__ __forceinline__ void fetch_x(double (&x)[NX][NR], const Args& a, int64_t k0, int kw,
                                        int64_t c0, int nc, int kb, int ks) {
#pragma unroll
  for (int h = 0; h < NX; ++h)
#pragma unroll
    for (int c = 0; c < NR; ++c) {
      const int k = kb + h * ks;
      x[h][c] = (k < kw && c < nc) ? ld_poll(a.X + (k0 + k) + (c0 + c) * a.ldx) : 0.0;
    }
}
// Re-read the entries still pending until the whole warp has them.
// Bounded: after kWaitNs the pending entries become NaN and the count of
// expired waits is raised; every other wait of the solve then gives up at
// once, so a lost block costs one bound, not one per block, and its NaN
// propagates to every later block (a failed solve never looks like a
// result).
template <int NX, int NR>
__device__ __forceinline__ void settle_x(double (&x)[NX][NR], const Args& a, int64_t k0,
                                         int64_t c0, int kb, int ks, int lane) {
  bool ok = true;
#pragma unroll
  for (int h = 0; h < NX; ++h)
#pragma unroll
    for (int c = 0; c < NR; ++c) ok &= !pending(x[h][c]);
  if (__all_sync(0xffffffffu, ok)) return;
  const unsigned long long t0 = global_ns();
  for (;;) {
    ok = true;
#pragma unroll
    for (int h = 0; h < NX; ++h)
#pragma unroll
      for (int c = 0; c < NR; ++c)
        if (pending(x[h][c])) {
          x[h][c] = ld_poll(a.X + (k0 + kb + h * ks) + (c0 + c) * a.ldx);
          ok &= !pending(x[h][c]);
        }
    if (__all_sync(0xffffffffu, ok)) return;
    const bool expired = global_ns() - t0 > a.wait_ns;
    if (__any_sync(0xffffffffu, expired || *(volatile unsigned*)(a.sync + 1) != 0u)) {
#pragma unroll
      for (int h = 0; h < NX; ++h)
#pragma unroll
        for (int c = 0; c < NR; ++c)
          if (pending(x[h][c])) x[h][c] = __longlong_as_double((long long)kQuietNaN);
      if (lane == 0 && expired) atomicAdd(a.sync + 1, 1u);
      return;
    }
  }
}

// One CTA per (row block, group): warps stream their shares of the tiles
// of all blocks but the previous one without CTA barriers; one barrier
// combines the partial sums into c = Dinv y; the hand-over x = c - W x_prev
// runs per warp (W = Dinv op(T)[block, previous block] in registers: rows
// 8 warp + i, columns lane and lane + 32).
template <bool TRANS, int NR, bool V16>
__global__ void __launch_bounds__(kThreads, 2)
trsv_kernel(Args a) {
  constexpr int PD = NR == 1 ? 3 : 2;     // tiles whose solution entries are fetched ahead
  constexpr int NX = TRANS ? 2 : 1;       // solution entries per lane per tile
  extern __shared__ __align__(16) unsigned char smem[];
  float* ring = reinterpret_cast<float*>(smem);
  double* Dinv = reinterpret_cast<double*>(smem + (size_t)S * 8 * kWarpTile * 4);
  float* Tw = reinterpret_cast<float*>(Dinv + BS * BS);
  double* part = reinterpret_cast<double*>(Tw + BS * BS);
  double* rdiag = part + 8 * NR * BS;
  int* ctrl = reinterpret_cast<int*>(rdiag + BS);

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) ctrl[0] = (int)atomicAdd(a.sync, 1u);
  __syncthreads();
  const int ticket = ctrl[0];
  const int t = ticket / a.ngroups, g = ticket - t * a.ngroups;
  const bool fwd = a.forward != 0;
  const int64_t r0 = (int64_t)(fwd ? t : a.nblk - 1 - t) * BS;
  const int rw = imin64(a.n - r0, BS);
  const int64_t c0 = (int64_t)g * NR;
  const int nc = imin64(a.nrhs - c0, NR);
  auto tile_k0 = [&](int q) -> int64_t { return (int64_t)(fwd ? q : a.nblk - 1 - q) * BS; };
  auto tile_kw = [&](int q) -> int { return imin64(a.n - tile_k0(q), BS); };
  const int nbulk = t > 1 ? t - 1 : 0;  // tiles before the previous block's
  // tile columns whose solution entries this lane reads in the bulk phase
  const int kb = TRANS ? lane : 8 * warp + (lane & 7);
  const int ks = TRANS ? 32 : 0;

  // ---- set-up copies: diagonal block, previous block's tile, ring prologue
  float* Dsrc = reinterpret_cast<float*>(Dinv);
  load_diag<V16>(Dsrc, a, r0, rw);
  if (t >= 1) load_tile<TRANS, V16>(Tw, a, r0, rw, tile_k0(t - 1), tile_kw(t - 1));
  cp_commit();
  float* wring = ring + warp * S * kWarpTile;
  auto issue = [&](int q) {
    if (q < nbulk)
      load_warp_tile<TRANS, V16>(wring + (q % S) * kWarpTile, a, r0, rw, tile_k0(q),
                                 tile_kw(q), warp, lane);
    cp_commit();
  };
#pragma unroll
  for (int q = 0; q < S - 1; ++q) issue(q);
  double xq[PD][NX][NR];
#pragma unroll
  for (int d = 0; d < PD; ++d)
    if (d < nbulk) fetch_x<NX, NR>(xq[d], a, tile_k0(d), tile_kw(d), c0, nc, kb, ks);
  // right-hand sides of rows lane and lane + 32
  double bm[2][NR];
#pragma unroll
  for (int h = 0; h < 2; ++h)
#pragma unroll
    for (int c = 0; c < NR; ++c) {
      const int r = lane + 32 * h;
      bm[h][c] = (r < rw && c < nc) ? a.B[(r0 + r) + (c0 + c) * a.n] : 0.0;
    }

  cp_wait<S - 1>();
  __syncthreads();
  invert_diag<TRANS>(Dsrc, Dinv, rdiag, rw, fwd, a.unit != 0);

  // ---- W = Dinv * op(T)[block, previous block] ----
  double W[8][2];
#pragma unroll
  for (int i = 0; i < 8; ++i) W[i][0] = W[i][1] = 0.0;
  if (t >= 1) {
#pragma unroll 2
    for (int m4 = 0; m4 < BS / 4; ++m4) {
      float tk[2][4];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int k = lane + 32 * h;
        if (!TRANS) {
          const float4 u = *reinterpret_cast<const float4*>(Tw + tile_index<false>(4 * m4, k));
          tk[h][0] = u.x; tk[h][1] = u.y; tk[h][2] = u.z; tk[h][3] = u.w;
        } else {
#pragma unroll
          for (int mm = 0; mm < 4; ++mm) tk[h][mm] = Tw[tile_index<true>(4 * m4 + mm, k)];
        }
      }
#pragma unroll
      for (int mm = 0; mm < 4; ++mm)
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          const double d = Dinv[(8 * warp + i) * BS + 4 * m4 + mm];
          W[i][0] = fma(d, (double)tk[0][mm], W[i][0]);
          W[i][1] = fma(d, (double)tk[1][mm], W[i][1]);
        }
    }
  }

  // ---- bulk: the tiles before the previous block's, per warp.
  // Transposed: rows 8 warp + i, per-lane partials over columns lane and
  // lane + 32.  Not transposed: columns 8 warp + j, per-lane partials of
  // rows lane and lane + 32 (the solution entry of column j broadcast from
  // lane j). ----
  constexpr int NA = TRANS ? 8 : 2;
  double acc[NA][NR];
#pragma unroll
  for (int i = 0; i < NA; ++i)
#pragma unroll
    for (int c = 0; c < NR; ++c) acc[i][c] = 0.0;
#pragma unroll 1
  for (int q = 0; q < nbulk; ++q) {
    double x[NX][NR];
#pragma unroll
    for (int h = 0; h < NX; ++h)
#pragma unroll
      for (int c = 0; c < NR; ++c) x[h][c] = xq[0][h][c];
#pragma unroll
    for (int d = 0; d + 1 < PD; ++d)
#pragma unroll
      for (int h = 0; h < NX; ++h)
#pragma unroll
        for (int c = 0; c < NR; ++c) xq[d][h][c] = xq[d + 1][h][c];
    if (q + PD < nbulk)
      fetch_x<NX, NR>(xq[PD - 1], a, tile_k0(q + PD), tile_kw(q + PD), c0, nc, kb, ks);
    settle_x<NX, NR>(x, a, tile_k0(q), c0, kb, ks, lane);
    cp_wait<S - 2>();
    __syncwarp();
    issue(q + S - 1);
    const float* Ts = wring + (q % S) * kWarpTile;
    if (TRANS) {
#pragma unroll
      for (int h = 0; h < NX; ++h) {
        const int k = lane + 32 * h;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          const double tv = (double)Ts[i * BS + k];
#pragma unroll
          for (int c = 0; c < NR; ++c) acc[i][c] = fma(tv, x[h][c], acc[i][c]);
        }
      }
    } else {
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        double xj[NR];
#pragma unroll
        for (int c = 0; c < NR; ++c) xj[c] = __shfl_sync(0xffffffffu, x[0][c], j);
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const double tv = (double)Ts[j * BS + lane + 32 * h];
#pragma unroll
          for (int c = 0; c < NR; ++c) acc[h][c] = fma(tv, xj[c], acc[h][c]);
        }
      }
    }
  }
  cp_wait<0>();

  // the previous block's solution: fetched now, waited for after c
  double xf[2][NR];
  if (t >= 1) fetch_x<2, NR>(xf, a, tile_k0(t - 1), tile_kw(t - 1), c0, nc, lane, 32);

  // ---- partial sums of the warps -> y = b - sum -> c = Dinv y ----
  if (TRANS) {
#pragma unroll
    for (int c = 0; c < NR; ++c) {
      double v[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) v[i] = acc[i][c];
      const double s = row_reduce(v, lane);
      if ((lane & 3) == 0) part[c * BS + 8 * warp + (lane >> 2)] = s;
    }
  } else {
#pragma unroll
    for (int c = 0; c < NR; ++c)
#pragma unroll
      for (int h = 0; h < 2; ++h) part[(warp * NR + c) * BS + lane + 32 * h] = acc[h][c];
  }
  __syncthreads();
  double cv[NR];
#pragma unroll
  for (int c = 0; c < NR; ++c) {
    double y[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int m = lane + 32 * h;
      double s;
      if (TRANS) {
        s = part[c * BS + m];
      } else {
        s = part[c * BS + m];
#pragma unroll
        for (int w = 1; w < 8; ++w) s += part[(w * NR + c) * BS + m];
      }
      y[h] = bm[h][c] - s;
    }
    double v[8];
#pragma unroll
    for (int i = 0; i < 8; ++i)
      v[i] = fma(Dinv[(8 * warp + i) * BS + lane + 32], y[1],
                 Dinv[(8 * warp + i) * BS + lane] * y[0]);
    cv[c] = row_reduce(v, lane);
  }

  // ---- hand-over: x = c - W x_prev once the previous block is out ----
  if (t >= 1) {
    settle_x<2, NR>(xf, a, tile_k0(t - 1), c0, lane, 32, lane);
#pragma unroll
    for (int c = 0; c < NR; ++c) {
      double v[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) v[i] = fma(W[i][1], xf[1][c], W[i][0] * xf[0][c]);
      cv[c] -= row_reduce(v, lane);
    }
  }
  const int ri = 8 * warp + (lane >> 2);
  if ((lane & 3) == 0 && ri < rw && ticket != a.withhold) {
#pragma unroll
    for (int c = 0; c < NR; ++c)
      if (c < nc) st_publish(a.X + (r0 + ri) + (c0 + c) * a.ldx, cv[c]);
  }
}

// B <- X and X <- pending, for the rows and columns of the solve; the first
// thread also clears the ticket counter and the expired-wait count.
__global__ void trsv_prepare_kernel(int64_t n, int64_t nrhs, double* __restrict__ X,
                                    int64_t ldx, double* __restrict__ B,
                                    unsigned* __restrict__ sync) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e == 0) {
    sync[0] = 0;
    sync[1] = 0;
  }
  if (e >= n * nrhs) return;
  const int64_t c = e / n, i = e - c * n;
  double* p = X + i + c * ldx;
  B[e] = *p;
  *p = __longlong_as_double((long long)kPending);
}

// ======================================================================
// Group kernel (groups of 4 or 8 right-hand sides).  Row blocks publish
// through a per-group counter of finished blocks (release / acquire at GPU
// scope); the solution blocks of finished blocks are staged through the
// CTA's cp.async ring together with the tiles, so a CTA that starts behind
// the solve front streams its backlog at memory speed.
// ======================================================================

constexpr int kGS = 4;                 // ring stages of the group kernel
constexpr int kSyncHeader = 4;         // ticket, abort, expired waits, spare

__host__ __device__ constexpr size_t group_smem_bytes(int nr) {
  return (size_t)kGS * BS * BS * 4        // fp32 tiles
         + (size_t)kGS * nr * BS * 8      // fp64 solution blocks of the tiles
         + (size_t)BS * BS * 8            // inverse of the diagonal block
         + (size_t)nr * BS * 8            // right-hand side / y
         + (size_t)BS * 8                 // reciprocals of the diagonal
         + 64;                            // control words
}

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(unsigned* p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Solution block of a tile: rows k0 .. k0+kw of the group's columns, the
// rest zero.  Async form: 16-byte copies through L2 (the block was written
// by another SM; L1 is bypassed).  Sync form: L2 loads.
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
__global__ void __launch_bounds__(kThreads, 1)
trsv_group_kernel(Args a) {
  extern __shared__ __align__(16) unsigned char smem[];
  float* Tr = reinterpret_cast<float*>(smem);
  double* Xr = reinterpret_cast<double*>(smem + (size_t)kGS * BS * BS * 4);
  double* Dinv = Xr + kGS * NR * BS;
  double* ybuf = Dinv + BS * BS;
  double* rdiag = ybuf + NR * BS;
  int* ctrl = reinterpret_cast<int*>(rdiag + BS);  // ticket, avail[2], give-up

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
  auto tile_k0 = [&](int q) -> int64_t { return (int64_t)(fwd ? q : a.nblk - 1 - q) * BS; };
  auto tile_kw = [&](int q) -> int { return imin64(a.n - tile_k0(q), BS); };

  // right-hand side rows of this block
  for (int e = tid; e < NR * BS; e += kThreads) {
    const int c = e / BS, r = e % BS;
    ybuf[e] = (c < nc && r < rw) ? a.X[(r0 + r) + (c0 + c) * a.ldx] : 0.0;
  }
  float* Dsrc = reinterpret_cast<float*>(Dinv);
  load_diag<V16>(Dsrc, a, r0, rw);
  cp_commit();
  int avail = ctrl[1];
  unsigned xbits = 0;
  auto issue = [&](int q) {
    if (q < t) {
      const int st = q % kGS;
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
  for (int q = 0; q < kGS - 1; ++q) issue(q);

  cp_wait<kGS - 1>();
  __syncthreads();
  invert_diag<TRANS>(Dsrc, Dinv, rdiag, rw, fwd, a.unit != 0);

  // ---- all tiles of the blocks solved before this one; warp w rows
  // 8w .. 8w+7, per-lane partials over columns lane and lane + 32 ----
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
            if (global_ns() - t0 > a.wait_ns) {
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
    const int st = q % kGS;
    cp_wait<kGS - 2>();
    if (!((xbits >> st) & 1u))
      load_x_sync<NR>(Xr + st * NR * BS, a, tile_k0(q), tile_kw(q), c0, nc);
    __syncthreads();
    issue(q + kGS - 1);
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
        a.X[(r0 + r) + (c0 + c) * a.ldx] = __longlong_as_double((long long)kQuietNaN);
    }
    return;
  }

  // ---- y = b - sum, then x = Dinv y (rows 8 warp + i, lanes over j) ----
#pragma unroll
  for (int c = 0; c < NR; ++c) {
    double v[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = acc[i][c];
    const double s = row_reduce(v, lane);
    if ((lane & 3) == 0) ybuf[c * BS + 8 * warp + (lane >> 2)] -= s;
  }
  __syncthreads();
  const int ri = 8 * warp + (lane >> 2);
#pragma unroll
  for (int c = 0; c < NR; ++c) {
    double v[8];
#pragma unroll
    for (int i = 0; i < 8; ++i)
      v[i] = fma(Dinv[(8 * warp + i) * BS + lane + 32], ybuf[c * BS + lane + 32],
                 Dinv[(8 * warp + i) * BS + lane] * ybuf[c * BS + lane]);
    const double x = row_reduce(v, lane);
    if ((lane & 3) == 0 && ri < rw && c < nc) a.X[(r0 + ri) + (c0 + c) * a.ldx] = x;
  }
  __syncthreads();
  if (tid == 0) st_release(done, (unsigned)(t + 1));
}

int group_width(int64_t nrhs) { return nrhs >= 8 ? 8 : nrhs >= 4 ? 4 : nrhs >= 2 ? 2 : 1; }

template <bool TRANS, int NR, bool V16>
lu_status launch_one(cudaStream_t st, const Args& a) {
  size_t smem;
  void (*fn)(Args);
  if constexpr (NR <= 2) {
    smem = warp_smem_bytes(NR);
    fn = trsv_kernel<TRANS, NR, V16>;
  } else {
    smem = group_smem_bytes(NR);
    fn = trsv_group_kernel<TRANS, NR, V16>;
  }
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
// scheduling.  kRC also sizes the partial sums (n x ceil(n / kRC) doubles)
// and with them the compiled-in scratch of lu_refine_static_c
// (LU_REFINE_STATIC_SCRATCH_BYTES, checked against refine's layout at
// n = LU_REFINE_STATIC_MAX_N by a CPU test): a smaller kRC needs a larger
// array.
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


// ---- residuals of several right-hand sides: R = B - op(A) X, columns in
// groups of kRG, A read once per group (fp64 arithmetic, each sum in a fixed
// order, so the result does not depend on scheduling).  maxes[3c .. 3c+2]
// receive max |r|, |x|, |b| of column c.
constexpr int kRG = 8;    // right-hand sides per group
constexpr int kRK = 64;   // rows of X staged per step (not transposed)

__device__ __forceinline__ void atomic_max_abs(unsigned long long* p, double v) {
  atomicMax(p, (unsigned long long)__double_as_longlong(fabs(v)));
}

// Not transposed: thread per row i, sums over k in order.
__global__ void __launch_bounds__(kT)
residual_multi_kernel(int64_t n, int64_t nrhs, const float* __restrict__ A, int64_t lda,
                      const double* __restrict__ B, int64_t ldb,
                      const double* __restrict__ X, int64_t ldx, double* __restrict__ R,
                      int64_t ldr, unsigned long long* __restrict__ maxes) {
  __shared__ double xs[kRK][kRG];
  const int tid = threadIdx.x, lane = tid & 31;
  const int64_t i = (int64_t)blockIdx.x * kT + tid;
  const int64_t c0 = (int64_t)blockIdx.y * kRG;
  const int nc = (int)((nrhs - c0) < kRG ? (nrhs - c0) : kRG);
  double acc[kRG];
#pragma unroll
  for (int c = 0; c < kRG; ++c) acc[c] = 0.0;
  const float* row = A + (i < n ? i : 0);
  for (int64_t k0 = 0; k0 < n; k0 += kRK) {
    const int kw = (int)((n - k0) < kRK ? (n - k0) : kRK);
    for (int e = tid; e < kRK * kRG; e += kT) {
      const int c = e / kRK, kk = e % kRK;
      xs[kk][c] = (kk < kw && c < nc) ? X[(k0 + kk) + (c0 + c) * ldx] : 0.0;
    }
    __syncthreads();
    if (i < n) {
      if (kw == kRK) {
#pragma unroll 8
        for (int kk = 0; kk < kRK; ++kk) {
          const double a = (double)row[(k0 + kk) * lda];
#pragma unroll
          for (int c = 0; c < kRG; ++c) acc[c] = fma(a, xs[kk][c], acc[c]);
        }
      } else {
        for (int kk = 0; kk < kw; ++kk) {
          const double a = (double)row[(k0 + kk) * lda];
#pragma unroll
          for (int c = 0; c < kRG; ++c) acc[c] = fma(a, xs[kk][c], acc[c]);
        }
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int c = 0; c < kRG; ++c) {
    double r = 0.0, x = 0.0, b = 0.0;
    if (i < n && c < nc) {
      b = B[i + (c0 + c) * ldb];
      x = X[i + (c0 + c) * ldx];
      r = b - acc[c];
      R[i + (c0 + c) * ldr] = r;
    }
    double m[3] = {fabs(r), fabs(x), fabs(b)};
#pragma unroll
    for (int q = 0; q < 3; ++q) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) m[q] = fmax(m[q], __shfl_xor_sync(0xffffffffu, m[q], o));
      if (lane == 0 && c < nc) atomic_max_abs(&maxes[3 * (c0 + c) + q], m[q]);
    }
  }
}

// Transposed: r_j = b_j - sum_i A[i, j] x_i.  Warp w of a CTA owns columns
// j0 + 4w .. j0 + 4w + 3 of A; lanes run over i (coalesced), each lane sums
// its rows in order, then a halving exchange over the 32 lanes leaves the
// (column, right-hand side) pair 4-column x 8-rhs index `lane` in lane.
constexpr int kTJ = 4;                 // columns of A per warp
constexpr int kTI = 256;               // rows of X staged per step
__global__ void __launch_bounds__(kT)
residual_multi_t_kernel(int64_t n, int64_t nrhs, const float* __restrict__ A, int64_t lda,
                        const double* __restrict__ B, int64_t ldb,
                        const double* __restrict__ X, int64_t ldx, double* __restrict__ R,
                        int64_t ldr, unsigned long long* __restrict__ maxes) {
  __shared__ double xs[kRG][kTI];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int64_t jb = (int64_t)blockIdx.x * (kT / 32) * kTJ + warp * kTJ;
  const int64_t c0 = (int64_t)blockIdx.y * kRG;
  const int nc = (int)((nrhs - c0) < kRG ? (nrhs - c0) : kRG);
  double v[kTJ * kRG];
#pragma unroll
  for (int q = 0; q < kTJ * kRG; ++q) v[q] = 0.0;
  for (int64_t i0 = 0; i0 < n; i0 += kTI) {
    const int iw = (int)((n - i0) < kTI ? (n - i0) : kTI);
    for (int e = tid; e < kTI * kRG; e += kT) {
      const int c = e / kTI, ii = e % kTI;
      xs[c][ii] = (ii < iw && c < nc) ? X[(i0 + ii) + (c0 + c) * ldx] : 0.0;
    }
    __syncthreads();
#pragma unroll
    for (int jj = 0; jj < kTJ; ++jj) {
      const int64_t j = jb + jj;
      if (j < n) {
        const float* col = A + j * lda + i0;
        for (int ii = lane; ii < iw; ii += 32) {
          const double a = (double)col[ii];
#pragma unroll
          for (int c = 0; c < kRG; ++c) v[jj * kRG + c] = fma(a, xs[c][ii], v[jj * kRG + c]);
        }
      }
    }
    __syncthreads();
  }
  // halving exchange: after the step with offset s, slot q holds index
  // q + (bits of lane above s) -- finally slot 0 holds index `lane`
#pragma unroll
  for (int s = 16; s >= 1; s >>= 1) {
    const bool up = lane & s;
#pragma unroll
    for (int q = 0; q < s; ++q) {
      const double send = up ? v[q] : v[q + s];
      const double keep = up ? v[q + s] : v[q];
      v[q] = keep + __shfl_xor_sync(0xffffffffu, send, s);
    }
  }
  const int jj = lane / kRG, c = lane % kRG;
  const int64_t j = jb + jj;
  if (j < n && c < nc) {
    const double b = B[j + (c0 + c) * ldb];
    const double x = X[j + (c0 + c) * ldx];
    const double r = b - v[0];
    R[j + (c0 + c) * ldr] = r;
    atomic_max_abs(&maxes[3 * (c0 + c)], r);
    atomic_max_abs(&maxes[3 * (c0 + c) + 1], x);
    atomic_max_abs(&maxes[3 * (c0 + c) + 2], b);
  }
}
}  // namespace

size_t trsm_sync_bytes(int64_t nrhs) {
  const int64_t groups = ceil_div(nrhs < 1 ? 1 : nrhs, 4);
  return align_up((size_t)(trsv::kSyncHeader + groups) * 4, 256);
}

size_t trsm_ws_bytes(int64_t n, int64_t nrhs) {
  return trsm_sync_bytes(nrhs) +
         align_up((size_t)(n < 0 ? 0 : n) * (size_t)(nrhs < 0 ? 0 : nrhs) * 8, 256);
}

lu_status launch_trsm(cudaStream_t st, int64_t n, const float* lu, int64_t ld,
                      double* X, int64_t ldx, int64_t nrhs, bool upper,
                      bool trans, unsigned* sync, double* B,
                      unsigned long long wait_ns, int withhold) {
  if (n <= 0 || nrhs <= 0) return LU_SUCCESS;
  if (!sync || !B) return LU_ERR_INVALID_ARG;
  const int nr = trsv::group_width(nrhs);
  if (ceil_div(n, trsv::BS) * ceil_div(nrhs, nr) > 0x7fffffffll) return LU_ERR_INVALID_ARG;
  trsv::Args a;
  a.lu = lu;
  a.ld = ld;
  a.X = X;
  a.ldx = ldx;
  a.B = B;
  a.n = n;
  a.nrhs = nrhs;
  a.nblk = (int)ceil_div(n, trsv::BS);
  a.ngroups = (int)ceil_div(nrhs, nr);
  // op(T) is lower (forward substitution) for L and for U^T
  a.forward = upper == trans;
  a.unit = !upper;
  a.xvec = ((reinterpret_cast<uintptr_t>(X) & 15) == 0) && (ldx % 2 == 0);
  a.sync = sync;
  a.wait_ns = wait_ns > 0 ? wait_ns : trsv::kWaitNs;
  a.withhold = withhold;
  if (nr <= 2) {
    const int64_t elems = n * nrhs;
    trsv::trsv_prepare_kernel<<<(unsigned)ceil_div(elems, 256), 256, 0, st>>>(n, nrhs, X, ldx,
                                                                            B, sync);
    LUB_LAUNCH_CHECK();
  } else {
    LUB_CUDA_TRY(cudaMemsetAsync(sync, 0, (size_t)(trsv::kSyncHeader + a.ngroups) * 4, st));
  }
  const bool v16 = ((reinterpret_cast<uintptr_t>(lu) & 15) == 0) && (ld % 4 == 0);
  if (trans)
    return v16 ? trsv::launch_nr<true, true>(st, a, nr) : trsv::launch_nr<true, false>(st, a, nr);
  return v16 ? trsv::launch_nr<false, true>(st, a, nr) : trsv::launch_nr<false, false>(st, a, nr);
}

lu_status launch_lu_solve(cudaStream_t st, int64_t n, const float* lu, int64_t ld,
                          double* X, int64_t ldx, int64_t nrhs, bool trans, unsigned* sync,
                          double* B) {
  if (!trans) {  // L U x = b: L y = b, then U x = y
    LUB_TRY(launch_trsm(st, n, lu, ld, X, ldx, nrhs, false, false, sync, B));
    return launch_trsm(st, n, lu, ld, X, ldx, nrhs, true, false, sync, B);
  }
  // (L U)^T x = U^T L^T x = b: U^T y = b, then L^T x = y
  LUB_TRY(launch_trsm(st, n, lu, ld, X, ldx, nrhs, true, true, sync, B));
  return launch_trsm(st, n, lu, ld, X, ldx, nrhs, false, true, sync, B);
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

lu_status launch_residual_multi(cudaStream_t st, int64_t n, int64_t nrhs, const float* A,
                                int64_t lda, const double* B, int64_t ldb, const double* X,
                                int64_t ldx, double* R, int64_t ldr, bool trans,
                                unsigned long long* maxes) {
  if (n <= 0 || nrhs <= 0) return LU_SUCCESS;
  LUB_CUDA_TRY(cudaMemsetAsync(maxes, 0, (size_t)3 * nrhs * sizeof(unsigned long long), st));
  const int64_t groups = ceil_div(nrhs, kRG);
  if (groups > 65535) return LU_ERR_INVALID_ARG;
  if (!trans) {
    dim3 g((unsigned)ceil_div(n, kT), (unsigned)groups);
    residual_multi_kernel<<<g, kT, 0, st>>>(n, nrhs, A, lda, B, ldb, X, ldx, R, ldr, maxes);
  } else {
    dim3 g((unsigned)ceil_div(n, (kT / 32) * kTJ), (unsigned)groups);
    residual_multi_t_kernel<<<g, kT, 0, st>>>(n, nrhs, A, lda, B, ldb, X, ldx, R, ldr, maxes);
  }
  LUB_LAUNCH_CHECK();
  return LU_SUCCESS;
}

lu_status launch_axpy(cudaStream_t st, int64_t n, const double* d, double* x) {
  axpy_kernel<<<(unsigned)ceil_div(n, 256), 256, 0, st>>>(n, d, x);
  LUB_LAUNCH_CHECK();
  return LU_SUCCESS;
}

}  // namespace lub
