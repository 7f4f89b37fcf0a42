// Tensor-core Schur update on sm_100a: C (fp32, column-major) -= A * B with
// A and B in fp16 / bf16 / e4m3, accumulated in fp32 in tensor memory.
//
// Replaces the reference's cublasGemmEx TC32 call for the trailing update
// (src/gemm.cu:255-287 called from src/lu_nopiv.hxx:172-183).
//
// Operand layouts (both K-major, what the tensor core consumes directly):
//   A : M x K, row-major        (row i at A + i*lda_p; the L21 copy)
//   B : K x N, column-major     (column j at B + j*ldb_p; the U12 copy)
// so a 128 x BK tile of A and a 256 x BK tile of B are each one TMA box of
// 128-byte rows with the 128-byte swizzle.
//
// One persistent CTA per SM, 10 warps:
//   warp 0      : TMA producer (4-stage ring of A/B tiles, mbarriers)
//   warp 1      : TMEM allocator + single-thread tcgen05.mma issuer
//                 (128 x 256 x 16 per instruction), commits to mbarriers
//   warps 2..9  : epilogue, two warpgroups; each warp owns 32 rows (its TMEM
//                 lane quarter) and 128 columns of the tile.  It reads the
//                 accumulator with tcgen05.ld in 32 x 32 chunks, writes
//                 scale * acc into a shared-memory staging tile and issues a
//                 TMA reduce-add of that tile into C, so C is updated in L2
//                 (one fp32 add, the same single rounding as C - acc) without
//                 the SM ever loading C -- or, in CTAs that stay for many
//                 tiles, streams C in by TMA ahead of the accumulator, adds in
//                 registers with the same roundings and stores it back by TMA.
//                 When C cannot be described by a tensor map (unaligned), the
//                 epilogue loads and stores C with ordinary coalesced accesses.
// Two TMEM accumulators (2 x 256 columns) let the epilogue of tile i overlap
// the MMAs of tile i+1.  Every mbarrier wait is bounded (sm100.cuh).
#include "common.cuh"
#include "kernels.cuh"
#include "sm100.cuh"
#include "tc_gemm.cuh"

#include <algorithm>
#include <cstring>
#include <mutex>
#include <type_traits>

namespace lub {
namespace {

using namespace sm100;

constexpr int BM = 128;
constexpr int BN = 256;
constexpr int kMaxSets = 8;  // operand sets summed in one pass
constexpr int kRowBytes = 128;                  // bytes of K per tile row
constexpr int kStageA = BM * kRowBytes;         // 16 KB
constexpr int kStageB = BN * kRowBytes;         // 32 KB
constexpr int kEpiWarps = 8;
constexpr int kThreads = 32 * (2 + kEpiWarps);  // 320
constexpr int kTmemCols = 2 * BN;               // two accumulators
constexpr int kEpiChunk = 32 * 32 * 4;          // one 32 x 32 fp32 staging tile

template <int EPI> struct Cfg;
template <> struct Cfg<0> {  // register epilogue
  static constexpr int kStages = 4;
  static constexpr size_t kEpiBytes = 0;
};
template <> struct Cfg<2> {  // register epilogue, fp16 C
  static constexpr int kStages = 4;
  static constexpr size_t kEpiBytes = 0;
};
template <> struct Cfg<1> {  // TMA reduce-add epilogue, 2 staging tiles per warp
  static constexpr int kStages = 3;
  static constexpr size_t kEpiBytes = (size_t)kEpiWarps * 2 * kEpiChunk;
};
template <> struct Cfg<3> {  // TMA load + store epilogue: each warp's 32 x 128 C block
  static constexpr int kStages = 2;
  static constexpr size_t kEpiBytes = (size_t)kEpiWarps * 4 * kEpiChunk;
};
template <> struct Cfg<4> {  // split K: the raw partial stored to its slab
  static constexpr int kStages = 4;
  static constexpr size_t kEpiBytes = 0;
};
template <int EPI>
constexpr size_t smem_bytes() {
  return 1024 /*align slack*/ + (size_t)Cfg<EPI>::kStages * (kStageA + kStageB) +
         Cfg<EPI>::kEpiBytes + 512;
}

__device__ __forceinline__ float to_f32(float x) { return x; }
__device__ __forceinline__ float to_f32(__half x) { return __half2float(x); }
template <typename T> __device__ __forceinline__ T from_f32(float x);
template <> __device__ __forceinline__ float from_f32<float>(float x) { return x; }
template <> __device__ __forceinline__ __half from_f32<__half>(float x) { return __float2half_rn(x); }

// Tensor maps of up to kMaxSets operand sets (A row-major, B column-major,
// both K-major), passed by value as one grid constant.
struct TcMaps {
  CUtensorMap a[kMaxSets];
  CUtensorMap b[kMaxSets];
};

struct TcParams {
  float* C;
  int64_t ldc;
  int M, N, K;
  int kb_count;        // number of BK blocks along K (all operand sets)
  int nsets;           // operand sets (1..kMaxSets): set s supplies the K
  int kb_end[kMaxSets];  // blocks [kb_end[s-1], kb_end[s]) from maps.a/b[s],
                       // several outer steps' products summed in one accumulator
  int tiles_m, tiles_n;
  const int* scale_a;  // per 128-row tile of A (log2), or null
  const int* scale_b;  // per 128-column tile of B (log2), or null
  float alpha;         // C += alpha * acc (alpha = -1 for the Schur update)
  int* err;
  int tiles_per_cta;   // 0: persistent (tile = blockIdx.x, += gridDim.x);
                       // > 0: CTA b owns the consecutive tiles [b*T, b*T+T)
  long long wait_cycles;  // bound of each barrier wait (kWaitCycles)
  int withhold;        // self-test of the give-up path only: the producer
                       // issues no loads, so every consumer wait runs out
  // split K (EPI 4): work unit u = tile u % tiles over the K blocks
  // [s kb_per, (s + 1) kb_per) of split s = u / tiles, whose raw fp32
  // product goes to slab s (part + s part_stride, column-major, part_ld);
  // ksplit = 1, kb_per = kb_count otherwise
  int ksplit, kb_per;
  float* part;
  int64_t part_ld, part_stride;
  int store;           // CTA pairs only: TMA store of alpha * acc (slab s at
                       // columns [s N, (s + 1) N) of tmap_c) instead of the
                       // reduce-add into C
};
// the update kernels take (TcMaps, CUtensorMap, TcParams, uint32_t) by value:
// within the 4 KB of kernel parameters
static_assert(sizeof(TcMaps) + sizeof(CUtensorMap) + sizeof(TcParams) + 16 <= 4096,
              "update kernel parameters exceed 4 KB");

// KIND 0: kind::f16 (fp16/bf16), 1: kind::f8f6f4 (e4m3).
// EPI  0: C loaded/stored by the epilogue threads; 1: TMA reduce-add;
//      2: as 0 with C stored in fp16 (C + alpha * acc in fp32, rounded once
//         to fp16; p.C then points at __half); 3: C streamed by TMA;
//      4: split K, the raw accumulator stored to the unit's slab.
template <int KIND, int EPI>
__global__ void __launch_bounds__(kThreads, 1)
tc_update_kernel(const __grid_constant__ TcMaps maps,
                 const __grid_constant__ CUtensorMap tmap_c, TcParams p,
                 uint32_t idesc) {
  constexpr int kStages = Cfg<EPI>::kStages;
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint8_t* sA = smem;
  uint8_t* sB = smem + kStages * kStageA;
  uint8_t* sEpi = sB + kStages * kStageB;
  uint64_t* full = reinterpret_cast<uint64_t*>(sEpi + Cfg<EPI>::kEpiBytes);
  uint64_t* empty = full + kStages;
  uint64_t* tfull = empty + kStages;
  uint64_t* tempty = tfull + 2;
  uint64_t* cfull = tempty + 2;  // EPI 3: four per epilogue warp
  uint64_t* drain = cfull + 4 * kEpiWarps;  // MMA completion after a give-up
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);

  const int warp = threadIdx.x / 32;
  const int lane = threadIdx.x % 32;
  // work units: tiles, times the K splits (unit == tile when ksplit == 1)
  const int num_tiles = p.tiles_m * p.tiles_n;
  const int num_units = num_tiles * p.ksplit;
  const int t_begin = p.tiles_per_cta > 0 ? (int)blockIdx.x * p.tiles_per_cta : (int)blockIdx.x;
  const int t_end = p.tiles_per_cta > 0 ? min(num_units, t_begin + p.tiles_per_cta) : num_units;
  const int t_step = p.tiles_per_cta > 0 ? 1 : (int)gridDim.x;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int a = 0; a < 2; ++a) {
      mbar_init(&tfull[a], 1);
      mbar_init(&tempty[a], kEpiWarps);
    }
    for (int w = 0; w < 4 * kEpiWarps; ++w) mbar_init(&cfull[w], 1);
    mbar_init(drain, 1);
    fence_barrier_init();
  }
  if (warp == 1) tmem_alloc(tmem_slot, kTmemCols);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;

  if (warp == 0) {
    // ---------------- TMA producer ----------------
    if (lane == 0) {
      for (int q = 0; q < p.nsets; ++q) {
        prefetch_tmap(&maps.a[q]);
        prefetch_tmap(&maps.b[q]);
      }
      int s = 0;
      uint32_t ph = 0;
      bool ok = !p.withhold;
      int armed = 0;
      for (int unit = t_begin; unit < t_end && ok; unit += t_step) {
        const int tile = unit % num_tiles;
        const int tm = tile % p.tiles_m, tn = tile / p.tiles_m;
        const int kb0 = (unit / num_tiles) * p.kb_per;
        const int kb1 = min(p.kb_count, kb0 + p.kb_per);
        int set = 0;
        for (int kb = kb0; kb < kb1; ++kb) {
          if (!mbar_wait(&empty[s], ph ^ 1, p.err, kErrTimeoutEmpty, p.wait_cycles)) {
            ok = false;
            break;
          }
          mbar_arrive_expect_tx(&full[s], kStageA + kStageB);
          while (kb >= p.kb_end[set]) ++set;
          const int kk = kb - (set > 0 ? p.kb_end[set - 1] : 0);
          const int kx = kk * kRowBytes;  // element offset along K == bytes for 8-bit
          const int kelem = KIND == 0 ? kk * (kRowBytes / 2) : kx;
          tma_load_2d(sA + s * kStageA, &maps.a[set], &full[s], kelem, tm * BM);
          tma_load_2d(sB + s * kStageB, &maps.b[set], &full[s], kelem, tn * BN);
          ++armed;
          if (++s == kStages) { s = 0; ph ^= 1; }
        }
      }
      if (!ok) {
        // a consumer may have given up before these loads landed: wait for
        // the last kStages armed stages (older ones were consumed) so no
        // copy into this CTA's shared memory outlives it
        int ss = s;
        uint32_t pp = ph;
        for (int j = 0; j < kStages && j < armed; ++j) {
          if (ss == 0) { ss = kStages - 1; pp ^= 1; } else { --ss; }
          mbar_drain(&full[ss], pp);
        }
      }
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer ----------------
    if (lane == 0) {
      int s = 0;
      uint32_t ph = 0;
      int local = 0;
      bool ok = true;
      bool issued = false;
      for (int unit = t_begin; unit < t_end && ok; unit += t_step, ++local) {
        const int acc = local & 1;
        const uint32_t aph = (local >> 1) & 1;
        const int kb0 = (unit / num_tiles) * p.kb_per;
        const int kb1 = min(p.kb_count, kb0 + p.kb_per);
        if (!mbar_wait(&tempty[acc], aph ^ 1, p.err, kErrTimeoutTmemEmpty, p.wait_cycles)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t d_tmem = tmem_base + acc * BN;
        for (int kb = kb0; kb < kb1; ++kb) {
          if (!mbar_wait(&full[s], ph, p.err, kErrTimeoutFull, p.wait_cycles)) {
            ok = false;
            break;
          }
          issued = true;
          tc_fence_after();
          const uint32_t a0 = smem_u32(sA + s * kStageA);
          const uint32_t b0 = smem_u32(sB + s * kStageB);
#pragma unroll
          for (int k = 0; k < 4; ++k) {  // 4 MMAs of 32 bytes of K each
            const uint64_t ad = sw128_kmajor_desc(a0 + k * 32);
            const uint64_t bd = sw128_kmajor_desc(b0 + k * 32);
            const uint32_t accum = (kb > kb0 || k > 0) ? 1u : 0u;
            if (KIND == 0) mma_f16(d_tmem, ad, bd, idesc, accum);
            else mma_f8(d_tmem, ad, bd, idesc, accum);
          }
          mma_commit(&empty[s]);  // frees the stage when these MMAs finish
          if (++s == kStages) { s = 0; ph ^= 1; }
        }
        if (ok) mma_commit(&tfull[acc]);
      }
      if (!ok && issued) {
        // MMAs still running read shared memory and write TMEM: wait for
        // all of them before the accumulator is freed
        mma_commit(drain);
        mbar_drain(drain, 0);
      }
    }
  } else {
    // ---------------- epilogue ----------------
    const int ew = warp - 2;             // 0..7
    const int quarter = warp & 3;        // TMEM lane quarter this warp may read
    const int half = ew / 4;             // columns [128*half, 128*half + 128)
    const int row_in_tile = quarter * 32 + lane;
    int local = 0;
    bool ok = true;
    if constexpr (EPI == 3) {
      // The warp's 32 x 128 block of C moves through four 32 x 32 chunk
      // buffers by TMA: chunk c of the next tile is loaded into buffer c as
      // soon as this tile's chunk c has been stored from it, so C streams in
      // ahead of the accumulator.  Each chunk gets s * acc added in
      // registers -- the product rounded, then the sum, as the reduce-add
      // epilogue rounds -- and goes back by TMA store.  Streaming C through
      // HBM this way runs faster than reductions performed in L2.
      float* cst = reinterpret_cast<float*>(sEpi + (size_t)ew * 4 * kEpiChunk);
      uint64_t* cb = cfull + ew * 4;
      uint32_t cph = 0;   // bit c: phase of buffer c
      uint32_t pend = 0;  // bit c: a load into buffer c not yet waited for
      auto valid = [&](int tile, int c) {
        const int tm = tile % p.tiles_m, tn = tile / p.tiles_m;
        return tm * BM + quarter * 32 < p.M && tn * BN + half * 128 + c * 32 < p.N;
      };
      auto load = [&](int tile, int c) {  // lane 0
        const int tm = tile % p.tiles_m, tn = tile / p.tiles_m;
        mbar_arrive_expect_tx(&cb[c], kEpiChunk);
        tma_load_2d(cst + c * (kEpiChunk / 4), &tmap_c, &cb[c], tm * BM + quarter * 32,
                    tn * BN + half * 128 + c * 32);
      };
      if (t_begin < t_end)
        for (int c = 0; c < 4; ++c)
          if (valid(t_begin, c)) {
            if (lane == 0) load(t_begin, c);
            pend |= 1u << c;
          }
      for (int tile = t_begin; tile < t_end && ok; tile += t_step, ++local) {
        const int tm = tile % p.tiles_m, tn = tile / p.tiles_m;
        const int acc = local & 1;
        const uint32_t aph = (local >> 1) & 1;
        const int col0 = tn * BN + half * 128;
        const int row0 = tm * BM + quarter * 32;
        const int next = tile + t_step;
        float sa = 1.0f;
        if (p.scale_a) sa = ldexpf(1.0f, -p.scale_a[tm]);
        if (!mbar_wait(&tfull[acc], aph, p.err, kErrTimeoutTmemFull, p.wait_cycles)) {
          ok = false;
          break;
        }
        tc_fence_after();
#pragma unroll 1
        for (int c = 0; c < 4; ++c) {
          const int cc = col0 + c * 32;
          const bool v = valid(tile, c);
          float av[32];
          const uint32_t taddr = tmem_base + ((uint32_t)(quarter * 32) << 16) +
                                 (uint32_t)(acc * BN + half * 128 + c * 32);
          tmem_ld32(taddr, av);
          tmem_ld_wait();
          if (c == 3) {  // accumulator fully read: hand it back to the MMA warp
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&tempty[acc]);
          }
          if (v) {
            if (!mbar_wait(&cb[c], (cph >> c) & 1u, p.err, kErrTimeoutFull, p.wait_cycles)) {
              ok = false;
              break;
            }
            cph ^= 1u << c;
            pend &= ~(1u << c);
            float sc = p.alpha * sa;
            if (p.scale_b) sc = ldexpf(sc, -p.scale_b[cc / 128]);
            float* box = cst + c * (kEpiChunk / 4);
#pragma unroll
            for (int j = 0; j < 32; ++j)
              box[j * 32 + lane] = __fadd_rn(box[j * 32 + lane], __fmul_rn(sc, av[j]));
            fence_proxy_async_smem();
            __syncwarp();
            if (lane == 0) {
              tma_store_2d(&tmap_c, box, row0, cc);
              bulk_commit_group();
            }
          }
          // buffer c, once read out by the store, takes chunk c of the next tile
          if (next < t_end && valid(next, c)) {
            if (lane == 0) {
              if (v) bulk_wait_group_read<0>();
              load(next, c);
            }
            pend |= 1u << c;
          }
        }
      }
      // every load was issued for a tile of this loop and waited for in it,
      // unless a bounded wait gave up: then wait for the loads still in flight
      if (lane == 0) {
        for (int c = 0; c < 4; ++c)
          if (pend & (1u << c)) mbar_drain(&cb[c], (cph >> c) & 1u);
        bulk_wait_group<0>();
      }
      __syncwarp();
    } else if constexpr (EPI == 1) {
      float* stage = reinterpret_cast<float*>(sEpi + (size_t)ew * 2 * kEpiChunk);
      int issued = 0;  // reduces issued by this warp; buffer = issued & 1
      for (int tile = t_begin; tile < t_end && ok; tile += t_step, ++local) {
        const int tm = tile % p.tiles_m, tn = tile / p.tiles_m;
        const int acc = local & 1;
        const uint32_t aph = (local >> 1) & 1;
        const int col0 = tn * BN + half * 128;
        float sa = 1.0f;
        if (p.scale_a) sa = ldexpf(1.0f, -p.scale_a[tm]);
        if (!mbar_wait(&tfull[acc], aph, p.err, kErrTimeoutTmemFull, p.wait_cycles)) {
          ok = false;
          break;
        }
        tc_fence_after();
#pragma unroll 1
        for (int c = 0; c < 4; ++c) {
          const int cc = col0 + c * 32;
          float av[32];
          const uint32_t taddr = tmem_base + ((uint32_t)(quarter * 32) << 16) +
                                 (uint32_t)(acc * BN + half * 128 + c * 32);
          tmem_ld32(taddr, av);
          tmem_ld_wait();
          if (c == 3) {  // accumulator fully read: hand it back to the MMA warp
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&tempty[acc]);
          }
          // whole 32 x 32 box outside C: nothing to add
          if (cc >= p.N || tm * BM + quarter * 32 >= p.M) continue;
          float s = p.alpha * sa;
          if (p.scale_b) s = ldexpf(s, -p.scale_b[cc / 128]);
          float* buf = stage + (issued & 1) * (kEpiChunk / 4);
          // the reduce issued two commits ago (same buffer) must be done
          // reading it; at most the latest one (other buffer) may remain
          if (lane == 0) bulk_wait_group_read<1>();
          __syncwarp();
#pragma unroll
          for (int j = 0; j < 32; ++j) buf[j * 32 + lane] = s * av[j];
          fence_proxy_async_smem();
          __syncwarp();
          if (lane == 0) {
            tma_reduce_add_2d(&tmap_c, buf, tm * BM + quarter * 32, cc);
            bulk_commit_group();
          }
          ++issued;
        }
      }
      if (lane == 0) bulk_wait_group<0>();
      __syncwarp();
    } else {
      using CT = typename std::conditional<EPI == 2, __half, float>::type;
      for (int unit = t_begin; unit < t_end && ok; unit += t_step, ++local) {
        const int tile = unit % num_tiles;
        const int tm = tile % p.tiles_m, tn = tile / p.tiles_m;
        const int acc = local & 1;
        const uint32_t aph = (local >> 1) & 1;
        const int64_t row = (int64_t)tm * BM + row_in_tile;
        const bool row_ok = row < p.M;
        const int col0 = tn * BN + half * 128;
        float sa = 1.0f;
        if (p.scale_a) sa = ldexpf(1.0f, -p.scale_a[tm]);
        // EPI 4: the unit's slab instead of C, nothing loaded
        const int64_t ldc = EPI == 4 ? p.part_ld : p.ldc;
        CT* cbase = (EPI == 4 ? reinterpret_cast<CT*>(p.part + (unit / num_tiles) * p.part_stride)
                              : reinterpret_cast<CT*>(p.C)) +
                    row + (int64_t)col0 * ldc;
        float cv[32];
        // load the first chunk of C before waiting for the accumulator
#pragma unroll
        for (int j = 0; j < 32; ++j)
          cv[j] = (EPI != 4 && row_ok && col0 + j < p.N) ? to_f32(cbase[j * ldc]) : 0.0f;
        if (!mbar_wait(&tfull[acc], aph, p.err, kErrTimeoutTmemFull, p.wait_cycles)) {
          ok = false;
          break;
        }
        tc_fence_after();
#pragma unroll 1
        for (int c = 0; c < 4; ++c) {
          CT* cp = cbase + (int64_t)(c * 32) * ldc;
          const int cc = col0 + c * 32;
          if (EPI != 4 && c > 0) {
#pragma unroll
            for (int j = 0; j < 32; ++j)
              cv[j] = (row_ok && cc + j < p.N) ? to_f32(cp[j * ldc]) : 0.0f;
          }
          float av[32];
          const uint32_t taddr = tmem_base + ((uint32_t)(quarter * 32) << 16) +
                                 (uint32_t)(acc * BN + half * 128 + c * 32);
          tmem_ld32(taddr, av);
          tmem_ld_wait();
          float s = p.alpha * sa;
          if (p.scale_b) s = ldexpf(s, -p.scale_b[cc / 128]);
#pragma unroll
          for (int j = 0; j < 32; ++j) {
            if (row_ok && cc + j < p.N) {
              if (EPI == 4) cp[j * ldc] = from_f32<CT>(av[j]);
              else cp[j * ldc] = from_f32<CT>(__fmaf_rn(s, av[j], cv[j]));
            }
          }
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&tempty[acc]);
      }
    }
  }

  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem_base, kTmemCols);
  }
}

// ---------------------------------------------------------------------------
// CTA-pair form for the large passes (fp16 / bf16 operands, fp32 C updated
// by TMA reduce-add): a cluster of two CTAs owns 256 x 256 tiles, and the
// even CTA issues tcgen05.mma.cta_group::2 (M = 256, N = 256) over both.
// Each CTA stages its own 128 rows of A and 128 columns of B per K block
// (32 KB, where a 128 x 256 tile alone needs 48 KB), so B crosses from L2
// once per 256 rows and five stages fit beside the epilogue buffers.  Both
// CTAs' copies count their bytes on the even CTA's `full` barrier; its
// commits arrive on the `empty` / `tfull` barriers of both CTAs; each CTA's
// epilogue reads its own accumulator rows and arrives on the even CTA's
// `tempty`.  Every element's products are accumulated in the same K order
// as by the single-CTA kernel.  No multicast loads: each CTA loads only
// what it stages itself.
constexpr int kPairRows = 128;                   // rows of A / columns of B per CTA
constexpr int kPairStage = kPairRows * kRowBytes;  // 16 KB each for A and B
constexpr int kPairStages = 5;
constexpr size_t kPairEpiBytes = (size_t)kEpiWarps * 2 * kEpiChunk;
constexpr size_t pair_smem_bytes() {
  return 1024 + (size_t)kPairStages * 2 * kPairStage + kPairEpiBytes + 512;
}

__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(kThreads, 1)
tc_update_pair_kernel(const __grid_constant__ TcMaps maps,
                      const __grid_constant__ CUtensorMap tmap_c, TcParams p,
                      uint32_t idesc) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint8_t* sA = smem;
  uint8_t* sB = smem + kPairStages * kPairStage;
  uint8_t* sEpi = sB + kPairStages * kPairStage;
  uint64_t* full = reinterpret_cast<uint64_t*>(sEpi + kPairEpiBytes);
  uint64_t* empty = full + kPairStages;
  uint64_t* tfull = empty + kPairStages;
  uint64_t* tempty = tfull + 2;
  uint64_t* drain = tempty + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);

  const uint32_t rank = cluster_ctarank();
  const bool leader = rank == 0;
  const int warp = threadIdx.x / 32;
  const int lane = threadIdx.x % 32;
  const int num_tiles = p.tiles_m * p.tiles_n;  // 256 x 256 tiles
  const int num_units = num_tiles * p.ksplit;    // x K ranges (split K)
  const int pair = (int)blockIdx.x >> 1;
  const int npairs = (int)gridDim.x >> 1;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kPairStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int a = 0; a < 2; ++a) {
      mbar_init(&tfull[a], 1);
      mbar_init(&tempty[a], 2 * kEpiWarps);  // both CTAs' epilogue warps
    }
    mbar_init(drain, 1);
    fence_barrier_init();
  }
  if (warp == 1) tmem_alloc_pair(tmem_slot, kTmemCols);
  tc_fence_before();
  cluster_sync();  // both CTAs' barriers initialised and tensor memory allocated
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;

  if (warp == 0) {
    // ---------------- TMA producer (both CTAs) ----------------
    if (lane == 0) {
      for (int q = 0; q < p.nsets; ++q) {
        prefetch_tmap(&maps.a[q]);
        prefetch_tmap(&maps.b[q]);
      }
      const uint32_t full0 = cluster_addr(&full[0], 0);  // the even CTA's barriers
      int s = 0;
      uint32_t ph = 0;
      bool ok = true;
      int armed = 0;
      for (int unit = pair; unit < num_units && ok; unit += npairs) {
        const int tile = unit % num_tiles;
        const int tm = tile % p.tiles_m, tn = tile / p.tiles_m;
        const int kb0 = (unit / num_tiles) * p.kb_per;
        const int kb1 = min(p.kb_count, kb0 + p.kb_per);
        int set = 0;
        for (int kb = kb0; kb < kb1; ++kb) {
          if (!mbar_wait(&empty[s], ph ^ 1, p.err, kErrTimeoutEmpty, p.wait_cycles)) {
            ok = false;
            break;
          }
          if (leader) mbar_arrive_expect_tx(&full[s], 4 * kPairStage);
          while (kb >= p.kb_end[set]) ++set;
          const int kelem = (kb - (set > 0 ? p.kb_end[set - 1] : 0)) * (kRowBytes / 2);
          const uint32_t bar = full0 + (uint32_t)(s * sizeof(uint64_t));
          tma_load_2d_pair(sA + s * kPairStage, &maps.a[set], bar, kelem,
                           tm * 2 * kPairRows + (int)rank * kPairRows);
          tma_load_2d_pair(sB + s * kPairStage, &maps.b[set], bar, kelem,
                           tn * 2 * kPairRows + (int)rank * kPairRows);
          ++armed;
          if (++s == kPairStages) { s = 0; ph ^= 1; }
        }
      }
      if (!ok && leader) {
        // the last stages' copies (both CTAs', counted here) must land
        // before this CTA's shared memory goes away
        int ss = s;
        uint32_t pp = ph;
        for (int j = 0; j < kPairStages && j < armed; ++j) {
          if (ss == 0) { ss = kPairStages - 1; pp ^= 1; } else { --ss; }
          mbar_drain(&full[ss], pp);
        }
      }
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer (even CTA) ----------------
    if (lane == 0 && leader) {
      int s = 0;
      uint32_t ph = 0;
      int local = 0;
      bool ok = true;
      bool issued = false;
      for (int unit = pair; unit < num_units && ok; unit += npairs, ++local) {
        const int acc = local & 1;
        const uint32_t aph = (local >> 1) & 1;
        const int kb0 = (unit / num_tiles) * p.kb_per;
        const int kb1 = min(p.kb_count, kb0 + p.kb_per);
        if (!mbar_wait(&tempty[acc], aph ^ 1, p.err, kErrTimeoutTmemEmpty, p.wait_cycles)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t d_tmem = tmem_base + acc * BN;
        for (int kb = kb0; kb < kb1; ++kb) {
          if (!mbar_wait(&full[s], ph, p.err, kErrTimeoutFull, p.wait_cycles)) {
            ok = false;
            break;
          }
          issued = true;
          tc_fence_after();
          const uint32_t a0 = smem_u32(sA + s * kPairStage);
          const uint32_t b0 = smem_u32(sB + s * kPairStage);
#pragma unroll
          for (int k = 0; k < 4; ++k)
            mma_f16_pair(d_tmem, sw128_kmajor_desc(a0 + k * 32), sw128_kmajor_desc(b0 + k * 32),
                         idesc, (kb > kb0 || k > 0) ? 1u : 0u);
          mma_commit_pair(&empty[s]);  // frees stage s in both CTAs
          if (++s == kPairStages) { s = 0; ph ^= 1; }
        }
        if (ok) mma_commit_pair(&tfull[acc]);
      }
      if (!ok && issued) {
        mma_commit_pair(drain);
        mbar_drain(drain, 0);
      }
    }
  } else {
    // ---------------- epilogue (both CTAs): TMA reduce-add ----------------
    const int ew = warp - 2;
    const int quarter = warp & 3;
    const int half = ew / 4;
    const uint32_t tempty0 = cluster_addr(&tempty[0], 0);
    float* stage = reinterpret_cast<float*>(sEpi + (size_t)ew * 2 * kEpiChunk);
    int issued = 0;
    int local = 0;
    for (int unit = pair; unit < num_units; unit += npairs, ++local) {
      const int tile = unit % num_tiles;
      const int tm = tile % p.tiles_m, tn = tile / p.tiles_m;
      const int acc = local & 1;
      const uint32_t aph = (local >> 1) & 1;
      const int row0 = tm * 2 * kPairRows + (int)rank * kPairRows + quarter * 32;
      const int col0 = tn * BN + half * 128;
      const int slab_col = (unit / num_tiles) * p.N;  // store mode: the unit's slab
      if (!mbar_wait(&tfull[acc], aph, p.err, kErrTimeoutTmemFull, p.wait_cycles)) break;
      tc_fence_after();
#pragma unroll 1
      for (int c = 0; c < 4; ++c) {
        const int cc = col0 + c * 32;
        float av[32];
        tmem_ld32(tmem_base + ((uint32_t)(quarter * 32) << 16) +
                      (uint32_t)(acc * BN + half * 128 + c * 32),
                  av);
        tmem_ld_wait();
        if (c == 3) {  // accumulator read out: hand it back to the even CTA
          tc_fence_before();
          __syncwarp();
          if (lane == 0)
            mbar_arrive_cluster(tempty0 + (uint32_t)(acc * sizeof(uint64_t)));
        }
        if (cc >= p.N || row0 >= p.M) continue;
        float* buf = stage + (issued & 1) * (kEpiChunk / 4);
        if (lane == 0) bulk_wait_group_read<1>();
        __syncwarp();
#pragma unroll
        for (int j = 0; j < 32; ++j) buf[j * 32 + lane] = p.alpha * av[j];
        fence_proxy_async_smem();
        __syncwarp();
        if (lane == 0) {
          if (p.store) tma_store_2d(&tmap_c, buf, row0, slab_col + cc);
          else tma_reduce_add_2d(&tmap_c, buf, row0, cc);
          bulk_commit_group();
        }
        ++issued;
      }
    }
    if (lane == 0) bulk_wait_group<0>();
    __syncwarp();
  }

  __syncwarp();
  tc_fence_before();
  cluster_sync();  // the peer has finished: no arrivals or copies into this CTA remain
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc_pair(tmem_base, kTmemCols);
  }
}

// ---------------------------------------------------------------------------
// host side: tensor maps through the driver entry point (no -lcuda)

using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t,
                                   void*, const cuuint64_t*, const cuuint64_t*,
                                   const cuuint32_t*, const cuuint32_t*,
                                   CUtensorMapInterleave, CUtensorMapSwizzle,
                                   CUtensorMapL2promotion,
                                   CUtensorMapFloatOOBfill);

EncodeTiledFn get_encode() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault,
                                &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  });
  return fn;
}

// rows x inner (inner contiguous, row stride ld elements), box box_rows x
// (128 bytes of inner).
// Column-major fp32 C (rows contiguous), 32 x 32 boxes, no swizzle.
bool make_c_map(CUtensorMap* map, float* C, int64_t M, int64_t N, int64_t ldc) {
  auto enc = get_encode();
  if (!enc) return false;
  cuuint64_t dims[2] = {(cuuint64_t)M, (cuuint64_t)N};
  cuuint64_t strides[1] = {(cuuint64_t)(ldc * 4)};
  cuuint32_t box[2] = {32, 32};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, C, dims, strides, box,
                   estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

bool make_kmajor_map(CUtensorMap* map, const void* base, CUtensorMapDataType dt,
                     int esize, int64_t inner, int64_t rows, int64_t ld,
                     int box_rows) {
  auto enc = get_encode();
  if (!enc) return false;
  cuuint64_t dims[2] = {(cuuint64_t)inner, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)(ld * esize)};
  cuuint32_t box[2] = {(cuuint32_t)(kRowBytes / esize), (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = enc(map, dt, 2, const_cast<void*>(base), dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

}  // namespace

namespace {
// persistent passes of at least this many 128 x 256 tiles run as CTA pairs
constexpr int kPairMinTiles = 2 * 148;

// Operand sets of one pass: set q is A[q] (M x K[q], row-major, lda_p) and
// B[q] (K[q] x N, column-major, ldb_p), summed in one accumulator.
struct OpSets {
  int n = 1;
  int64_t K[kMaxSets] = {};
  const void* A[kMaxSets] = {};
  const void* B[kMaxSets] = {};
};

OpSets one_set(int64_t K, const void* A, const void* B) {
  OpSets o;
  o.K[0] = K;
  o.A[0] = A;
  o.B[0] = B;
  return o;
}

// Checks the sets and encodes their tensor maps (box_rows_a / box_rows_b
// rows per box); fills kb_count / nsets / kb_end.
lu_status encode_sets(const OpSets& ops, TcOperand kind, int64_t M, int64_t N, int64_t lda_p,
                      int64_t ldb_p, int box_rows_a, int box_rows_b, TcMaps* maps,
                      TcParams* p) {
  if (ops.n < 1 || ops.n > kMaxSets) return LU_ERR_INVALID_ARG;
  const int esize = (kind == TcOperand::E4M3) ? 1 : 2;
  if ((lda_p * esize) % 16 != 0 || (ldb_p * esize) % 16 != 0) return LU_ERR_INVALID_ARG;
  // split copies are plain fp16 operands with a tripled K
  const CUtensorMapDataType dt = kind == TcOperand::BF16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16
                               : kind == TcOperand::E4M3 ? CU_TENSOR_MAP_DATA_TYPE_UINT8
                                                         : CU_TENSOR_MAP_DATA_TYPE_FLOAT16;
  std::memset(maps, 0, sizeof(*maps));
  int kb = 0;
  int64_t ksum = 0;
  for (int q = 0; q < ops.n; ++q) {
    const int64_t K = ops.K[q];
    if (K <= 0 || K > INT32_MAX || lda_p < K || ldb_p < K || !ops.A[q] || !ops.B[q] ||
        (uintptr_t)ops.A[q] % 16 != 0 || (uintptr_t)ops.B[q] % 16 != 0)
      return LU_ERR_INVALID_ARG;
    if (!make_kmajor_map(&maps->a[q], ops.A[q], dt, esize, K, M, lda_p, box_rows_a) ||
        !make_kmajor_map(&maps->b[q], ops.B[q], dt, esize, K, N, ldb_p, box_rows_b))
      return LU_ERR_CUDA;
    kb += (int)ceil_div(K * esize, kRowBytes);
    ksum += K;
    p->kb_end[q] = kb;
  }
  for (int q = ops.n; q < kMaxSets; ++q) p->kb_end[q] = kb;
  if (ksum > INT32_MAX) return LU_ERR_INVALID_ARG;
  p->nsets = ops.n;
  p->kb_count = kb;
  p->K = (int)ksum;
  return LU_SUCCESS;
}

lu_status tc_update_pair_impl(cudaStream_t st, TcOperand kind, int64_t M, int64_t N,
                              const OpSets& ops, int64_t lda_p, int64_t ldb_p, float* C,
                              int64_t ldc, float alpha, int* err, int max_ctas,
                              float* part = nullptr, int ksplit = 1, int* nslabs = nullptr);
int pair_capacity();

lu_status tc_update_impl(cudaStream_t st, TcOperand kind, int64_t M, int64_t N,
                         const OpSets& ops, float alpha, int64_t lda_p, int64_t ldb_p,
                         void* C, bool c_half, int64_t ldc, const int* scale_a,
                         const int* scale_b, int* err, int max_ctas, int tiles_per_cta,
                         long long wait_cycles = 0, int withhold = 0, int ksplit = 1,
                         float* part = nullptr) {
  if (M <= 0 || N <= 0 || ops.K[0] <= 0) return LU_SUCCESS;
  if (M > INT32_MAX || N > INT32_MAX) return LU_ERR_INVALID_ARG;
  if (ops.n > 1 && (scale_a || scale_b)) return LU_ERR_INVALID_ARG;
  TcParams p;
  std::memset(&p, 0, sizeof(p));
  TcMaps maps;
  LUB_TRY(encode_sets(ops, kind, M, N, lda_p, ldb_p, BM, BN, &maps, &p));
  p.C = static_cast<float*>(C);
  p.ldc = ldc;
  p.M = (int)M;
  p.N = (int)N;
  p.tiles_m = (int)ceil_div(M, BM);
  p.tiles_n = (int)ceil_div(N, BN);
  p.scale_a = scale_a;
  p.scale_b = scale_b;
  p.alpha = alpha;
  p.err = err;
  p.tiles_per_cta = tiles_per_cta;
  p.wait_cycles = wait_cycles > 0 ? wait_cycles : sm100::kWaitCycles;
  p.withhold = withhold ? 1 : 0;
  // split K: every split non-empty, one unit per CTA (the block scheduler
  // then interleaves concurrent launches' units)
  p.kb_per = p.kb_count;
  p.ksplit = 1;
  p.part = nullptr;
  p.part_ld = p.part_stride = 0;
  if (part) {
    if (ksplit < 1 || ops.n > 1 || scale_a || scale_b || c_half) return LU_ERR_INVALID_ARG;
    p.kb_per = (int)ceil_div(p.kb_count, ksplit);
    p.ksplit = (int)ceil_div(p.kb_count, p.kb_per);
    p.part = part;
    p.part_ld = (M + 3) / 4 * 4;
    p.part_stride = p.part_ld * N;
    tiles_per_cta = 1;
  }
  const int tiles = p.tiles_m * p.tiles_n * p.ksplit;
  const int grid = tiles_per_cta > 0
                       ? (int)ceil_div(tiles, tiles_per_cta)
                       : std::min(tiles, max_ctas > 0 ? max_ctas : sm_count());
  // TMA reduce-add needs a 16-byte aligned C with a 16-byte multiple stride
  CUtensorMap mc;
  std::memset(&mc, 0, sizeof(mc));
  const bool tma_c = !part && !c_half && ((uintptr_t)C % 16 == 0) && (ldc % 4 == 0) &&
                     make_c_map(&mc, static_cast<float*>(C), M, N, ldc);
  // C epilogue: CTAs that stay for many tiles stream C by TMA load / store,
  // its loads running ahead of the accumulator (B200, 16128^2 x 256:
  // 5.6 TB/s against 4.7 for the L2 reduce-add); CTAs of one or two tiles --
  // the trailing updates under look-ahead, which hand SMs back to the panel
  // kernels quickly -- have no pipeline to fill and keep the reduce-add.
  // With more than four 128-byte operand blocks along K (K = 512 at fp16:
  // two outer steps per pass) the operand feed bounds the tile, and the reduce-add
  // epilogue's smaller shared-memory footprint leaves room for a third
  // operand stage: 15360^2 x 512, 0.408 ms against 0.457 streaming C.
  const bool stream_c = (tiles_per_cta <= 0 || tiles_per_cta > 2) && p.kb_count <= 4;
  // large persistent passes with unscaled 16-bit operands and K >= 512:
  // CTA pairs (B200, 15360^2: K = 1024 0.473 ms against 0.563, K = 512 in
  // the factorization's bulk passes 2-3% faster; at K = 256 the streaming
  // epilogue of the single-CTA kernel wins, 0.375 against 0.474 ms)
  if (tma_c && !part && tiles_per_cta <= 0 && !withhold && !scale_a && !scale_b &&
      (kind == TcOperand::F16 || kind == TcOperand::BF16) && tiles >= kPairMinTiles &&
      p.kb_count >= 8 && pair_capacity() > 0)
    return tc_update_pair_impl(st, kind, M, N, ops, lda_p, ldb_p, static_cast<float*>(C), ldc,
                               alpha, err, max_ctas);
  const uint32_t f = kind == TcOperand::BF16 ? 1u : 0u;
  const uint32_t idesc = sm100::make_idesc(f, f, BM, BN);
  if (part) {
    if (kind != TcOperand::F16 && kind != TcOperand::BF16) return LU_ERR_UNSUPPORTED;
    LUB_CUDA_TRY(set_smem_limit((const void*)tc_update_kernel<0, 4>, smem_bytes<4>()));
    tc_update_kernel<0, 4><<<grid, kThreads, smem_bytes<4>(), st>>>(maps, mc, p, idesc);
  } else if (c_half) {
    if (kind != TcOperand::F16 && kind != TcOperand::BF16) return LU_ERR_UNSUPPORTED;
    LUB_CUDA_TRY(set_smem_limit((const void*)tc_update_kernel<0, 2>, smem_bytes<2>()));
    tc_update_kernel<0, 2><<<grid, kThreads, smem_bytes<2>(), st>>>(maps, mc, p, idesc);
  } else if (kind == TcOperand::E4M3) {
    if (tma_c && !stream_c) {
      LUB_CUDA_TRY(set_smem_limit((const void*)tc_update_kernel<1, 1>, smem_bytes<1>()));
      tc_update_kernel<1, 1><<<grid, kThreads, smem_bytes<1>(), st>>>(maps, mc, p, idesc);
    } else if (tma_c) {
      LUB_CUDA_TRY(set_smem_limit((const void*)tc_update_kernel<1, 3>, smem_bytes<3>()));
      tc_update_kernel<1, 3><<<grid, kThreads, smem_bytes<3>(), st>>>(maps, mc, p, idesc);
    } else {
      LUB_CUDA_TRY(set_smem_limit((const void*)tc_update_kernel<1, 0>, smem_bytes<0>()));
      tc_update_kernel<1, 0><<<grid, kThreads, smem_bytes<0>(), st>>>(maps, mc, p, idesc);
    }
  } else {
    if (tma_c && !stream_c) {
      LUB_CUDA_TRY(set_smem_limit((const void*)tc_update_kernel<0, 1>, smem_bytes<1>()));
      tc_update_kernel<0, 1><<<grid, kThreads, smem_bytes<1>(), st>>>(maps, mc, p, idesc);
    } else if (tma_c) {
      LUB_CUDA_TRY(set_smem_limit((const void*)tc_update_kernel<0, 3>, smem_bytes<3>()));
      tc_update_kernel<0, 3><<<grid, kThreads, smem_bytes<3>(), st>>>(maps, mc, p, idesc);
    } else {
      LUB_CUDA_TRY(set_smem_limit((const void*)tc_update_kernel<0, 0>, smem_bytes<0>()));
      tc_update_kernel<0, 0><<<grid, kThreads, smem_bytes<0>(), st>>>(maps, mc, p, idesc);
    }
  }
  LUB_LAUNCH_CHECK();
  return LU_SUCCESS;
}

// Clusters of two tc_update_pair_kernel CTAs resident at once on this
// device (cached per device; 0 if the query fails).
int pair_capacity() {
  static int cache[64];
  static std::once_flag once[64];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 0;
  std::call_once(once[dev], [dev] {
    cache[dev] = 0;
    // the query needs the kernel's shared-memory limit raised first
    if (set_smem_limit((const void*)tc_update_pair_kernel, pair_smem_bytes()) != cudaSuccess) {
      cudaGetLastError();
      return;
    }
    cudaLaunchConfig_t cfg;
    std::memset(&cfg, 0, sizeof(cfg));
    cfg.gridDim = dim3(2 * 148, 1, 1);
    cfg.blockDim = dim3(kThreads, 1, 1);
    cfg.dynamicSmemBytes = pair_smem_bytes();
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, (const void*)tc_update_pair_kernel, &cfg) !=
        cudaSuccess) {
      cudaGetLastError();
      n = 0;
    }
    cache[dev] = n;
  });
  return cache[dev];
}

// With part != nullptr: split-K partials instead of the update -- the K
// blocks cut into `ksplit` near-equal ranges, unit (tile, range s) stores
// its raw product by TMA into slab s of `part` (ld round4(M), slabs
// round4(M) x N apart); *nslabs receives the number of ranges.
lu_status tc_update_pair_impl(cudaStream_t st, TcOperand kind, int64_t M, int64_t N,
                              const OpSets& ops, int64_t lda_p, int64_t ldb_p, float* C,
                              int64_t ldc, float alpha, int* err, int max_ctas,
                              float* part, int ksplit, int* nslabs) {
  if (kind != TcOperand::F16 && kind != TcOperand::BF16) return LU_ERR_UNSUPPORTED;
  if (part) {
    C = part;
    ldc = (M + 3) / 4 * 4;
  }
  if ((uintptr_t)C % 16 != 0 || ldc % 4 != 0) return LU_ERR_INVALID_ARG;  // TMA reduce-add
  TcParams p;
  std::memset(&p, 0, sizeof(p));
  TcMaps maps;
  LUB_TRY(encode_sets(ops, kind, M, N, lda_p, ldb_p, kPairRows, kPairRows, &maps, &p));
  p.ksplit = 1;
  p.kb_per = p.kb_count;
  if (part) {
    if (ksplit < 1 || ops.n != 1) return LU_ERR_INVALID_ARG;
    p.kb_per = (int)ceil_div(p.kb_count, ksplit);
    p.ksplit = (int)ceil_div(p.kb_count, p.kb_per);
    p.store = 1;
    if (nslabs) *nslabs = p.ksplit;
  }
  CUtensorMap mc;
  if (!make_c_map(&mc, C, M, part ? N * p.ksplit : N, ldc)) return LU_ERR_CUDA;
  p.C = C;
  p.ldc = ldc;
  p.M = (int)M;
  p.N = (int)N;
  p.tiles_m = (int)ceil_div(M, 2 * kPairRows);
  p.tiles_n = (int)ceil_div(N, BN);
  p.alpha = alpha;
  p.err = err;
  p.wait_cycles = sm100::kWaitCycles;
  const int tiles = p.tiles_m * p.tiles_n * p.ksplit;
  LUB_CUDA_TRY(set_smem_limit((const void*)tc_update_pair_kernel, pair_smem_bytes()));
  // never more pairs than can be resident at once (SM pairs sit inside one
  // GPC, so an odd SM per GPC stays out): a pair scheduled late would run
  // its whole share of the tiles after the others
  const int resident = pair_capacity();
  if (resident < 1) return LU_ERR_UNSUPPORTED;
  const int pairs =
      std::max(1, std::min({tiles, (max_ctas > 0 ? max_ctas : sm_count()) / 2, resident}));
  const uint32_t f = kind == TcOperand::BF16 ? 1u : 0u;
  const uint32_t idesc = sm100::make_idesc(f, f, 2 * kPairRows, BN);
  tc_update_pair_kernel<<<2 * pairs, kThreads, pair_smem_bytes(), st>>>(maps, mc, p, idesc);
  LUB_LAUNCH_CHECK();
  return LU_SUCCESS;
}

}  // namespace

lu_status launch_tc_update(cudaStream_t st, TcOperand kind, int64_t M,
                           int64_t N, int64_t K, float alpha, const void* A,
                           int64_t lda_p, const void* B, int64_t ldb_p, float* C,
                           int64_t ldc, const int* scale_a, const int* scale_b,
                           int* err, int max_ctas, int tiles_per_cta) {
  return tc_update_impl(st, kind, M, N, one_set(K, A, B), alpha, lda_p, ldb_p, C, false, ldc,
                        scale_a, scale_b, err, max_ctas, tiles_per_cta);
}

lu_status launch_tc_update_sets(cudaStream_t st, TcOperand kind, int64_t M, int64_t N,
                                int nsets, const int64_t* K, const void* const* A,
                                const void* const* B, int64_t ld_p, float* C, int64_t ldc,
                                int* err, int max_ctas, int tiles_per_cta) {
  if (kind != TcOperand::F16 && kind != TcOperand::BF16) return LU_ERR_UNSUPPORTED;
  if (nsets < 1 || nsets > kMaxSets || !K || !A || !B) return LU_ERR_INVALID_ARG;
  OpSets o;
  o.n = nsets;
  for (int q = 0; q < nsets; ++q) {
    o.K[q] = K[q];
    o.A[q] = A[q];
    o.B[q] = B[q];
  }
  return tc_update_impl(st, kind, M, N, o, -1.0f, ld_p, ld_p, C, false, ldc, nullptr, nullptr,
                        err, max_ctas, tiles_per_cta);
}

lu_status launch_tc_update2(cudaStream_t st, TcOperand kind, int64_t M, int64_t N,
                            int64_t K, const void* A, const void* B, int64_t K2,
                            const void* A2, const void* B2, int64_t ld_p, float* C,
                            int64_t ldc, int* err, int max_ctas, int tiles_per_cta) {
  const int64_t ks[2] = {K, K2};
  const void* as[2] = {A, A2};
  const void* bs[2] = {B, B2};
  return launch_tc_update_sets(st, kind, M, N, K2 > 0 ? 2 : 1, ks, as, bs, ld_p, C, ldc, err,
                               max_ctas, tiles_per_cta);
}

lu_status launch_tc_update_h(cudaStream_t st, TcOperand kind, int64_t M, int64_t N,
                             int64_t K, float alpha, const void* A, int64_t lda_p,
                             const void* B, int64_t ldb_p, __half* C, int64_t ldc,
                             int* err) {
  return tc_update_impl(st, kind, M, N, one_set(K, A, B), alpha, lda_p, ldb_p, C, true, ldc,
                        nullptr, nullptr, err, 0, 0);
}

// C = rn(C + alpha * (part_0 + part_1 + ... + part_{S-1})), the partial
// sums added in split order (deterministic), the product scaled and added
// with one fma as in the unsplit epilogue; shadow (if given) receives the
// stored value widened to fp32.
template <typename CT>
__global__ void __launch_bounds__(256)
splitk_finish_kernel(int64_t M, int S, const float* __restrict__ part, int64_t part_ld,
                     int64_t part_stride, float alpha, CT* __restrict__ C, int64_t ldc,
                     float* __restrict__ shadow, int64_t lds) {
  const int64_t i = (int64_t)blockIdx.x * 256 + threadIdx.x;
  const int64_t j = blockIdx.y;
  if (i >= M) return;
  const float* q = part + i + j * part_ld;
  float t = q[0];
  for (int s = 1; s < S; ++s) t = __fadd_rn(t, q[s * part_stride]);
  CT& c = C[i + j * ldc];
  const CT v = from_f32<CT>(__fmaf_rn(alpha, t, to_f32(c)));
  c = v;
  if (shadow) shadow[i + j * lds] = to_f32(v);
}

int64_t splitk_slab_floats(int64_t M, int64_t N) { return (M + 3) / 4 * 4 * N; }

lu_status launch_tc_partials(cudaStream_t st, TcOperand kind, int64_t M, int64_t N,
                             int64_t K, const void* A, int64_t lda_p, const void* B,
                             int64_t ldb_p, int ksplit, float* part, int slab0, int* nslabs,
                             int* err) {
  if (nslabs) *nslabs = 0;
  if (M <= 0 || N <= 0 || K <= 0) return LU_SUCCESS;
  if (!part || ksplit < 1 || slab0 < 0) return LU_ERR_INVALID_ARG;
  float* base = part + (int64_t)slab0 * splitk_slab_floats(M, N);
  // 16-bit operands with at least 8 K blocks: CTA pairs storing their
  // partials by TMA (256 x 256 tiles: the split re-chosen for pairs).  The
  // slabs sit side by side as one tensor of N x S columns, so N must be a
  // multiple of the 32-column box (no box may reach into the next slab).
  const int64_t kbs = ceil_div(K * tc_operand_bytes(kind), kRowBytes);
  if ((kind == TcOperand::F16 || kind == TcOperand::BF16) && kbs >= 8 && N % 32 == 0 &&
      pair_capacity() > 0 &&
      (M + 3) / 4 * 4 * N * (int64_t)ksplit < INT32_MAX) {
    const int64_t tiles2 = ceil_div(M, 2 * kPairRows) * ceil_div(N, BN);
    const int ks2 = std::min(ksplit, tc_split_choice(tiles2, K, 2, pair_capacity(), ksplit));
    return tc_update_pair_impl(st, kind, M, N, one_set(K, A, B), lda_p, ldb_p, nullptr, 0, 1.0f,
                               err, 0, base, ks2, nslabs);
  }
  LUB_TRY(tc_update_impl(st, kind, M, N, one_set(K, A, B), 1.0f, lda_p, ldb_p, nullptr, false,
                         M, nullptr, nullptr, err, 0, 0, 0, 0, ksplit,
                         part + (int64_t)slab0 * splitk_slab_floats(M, N)));
  const int kb = (int)ceil_div(K * tc_operand_bytes(kind), kRowBytes);
  const int per = (int)ceil_div(kb, ksplit);
  if (nslabs) *nslabs = (int)ceil_div(kb, per);
  return LU_SUCCESS;
}

lu_status launch_splitk_finish(cudaStream_t st, int64_t M, int64_t N, int S, const float* part,
                               float alpha, void* C, bool c_half, int64_t ldc, float* shadow,
                               int64_t lds) {
  if (M <= 0 || N <= 0) return LU_SUCCESS;
  if (S < 1 || !part || N > 65535 || (shadow && lds < M)) return LU_ERR_INVALID_ARG;
  const int64_t pld = (M + 3) / 4 * 4;
  dim3 grid((unsigned)ceil_div(M, 256), (unsigned)N);
  if (c_half)
    splitk_finish_kernel<__half><<<grid, 256, 0, st>>>(M, S, part, pld, pld * N, alpha,
                                                        static_cast<__half*>(C), ldc, shadow,
                                                        lds);
  else
    splitk_finish_kernel<float><<<grid, 256, 0, st>>>(M, S, part, pld, pld * N, alpha,
                                                       static_cast<float*>(C), ldc, shadow,
                                                       lds);
  LUB_LAUNCH_CHECK();
  return LU_SUCCESS;
}

lu_status launch_tc_update_split(cudaStream_t st, TcOperand kind, int64_t M, int64_t N,
                                 int64_t K, float alpha, const void* A, int64_t lda_p,
                                 const void* B, int64_t ldb_p, void* C, bool c_half,
                                 int64_t ldc, float* shadow, int64_t lds, int ksplit,
                                 float* part, int* err) {
  if (M <= 0 || N <= 0 || K <= 0) return LU_SUCCESS;
  int S = 0;
  LUB_TRY(launch_tc_partials(st, kind, M, N, K, A, lda_p, B, ldb_p, ksplit, part, 0, &S, err));
  return launch_splitk_finish(st, M, N, S, part, alpha, C, c_half, ldc, shadow, lds);
}

int tc_split_choice(int64_t tiles, int64_t K, int esize, int sms, int smax) {
  const int64_t kb = ceil_div(K * esize, kRowBytes);
  int best = 1;
  double best_t = 0.0;
  for (int s = 1; s <= smax; ++s) {
    const int64_t per = ceil_div(kb, (int64_t)s);
    if (s > 1 && per < 4) break;  // at least K = 256 (fp16) per split
    const int64_t waves = ceil_div(tiles * s, (int64_t)sms);
    // a split costs a little extra (the partial written and summed)
    const double t = (double)waves * (double)per * (1.0 + 0.02 * (s - 1));
    if (s == 1 || t < best_t) {
      best = s;
      best_t = t;
    }
  }
  return best;
}

lu_status launch_tc_update_withheld(cudaStream_t st, int64_t M, int64_t N, int64_t K,
                                    const void* A, int64_t lda_p, const void* B,
                                    int64_t ldb_p, float* C, int64_t ldc, int* err,
                                    long long wait_cycles, int tiles_per_cta) {
  if (wait_cycles <= 0) return LU_ERR_INVALID_ARG;
  return tc_update_impl(st, TcOperand::F16, M, N, one_set(K, A, B), -1.0f, lda_p, ldb_p, C,
                        false, ldc, nullptr, nullptr, err, 0, tiles_per_cta, wait_cycles, 1);
}

}  // namespace lub
