// Right-looking driver for the in-place no-pivot LU.
//
// Reference structure (src/lu_nopiv.hxx:130-197 with the inner loop of
// src/lu_nopiv_inner_rl.hxx:104-196): for every outer block of nb columns,
// factor the block column and the block row with ib = 8 steps, then apply the
// trailing update with K = nb.
//
// Here each outer block column is processed in sub-panels of width
// diag_w <= 128:
//   diag_factor (1 CTA)  ->  lpanel (rows below) + upanel (columns right)
//   -> rank-8-chunked updates of the rest of the outer block column / row
// and the outer block finishes with one trailing update of K = nb.  Every
// element receives the same sequence of floating-point operations as in the
// reference loop, so the FP32 path equals the CPU restatement bit for bit.
#include "common.cuh"
#include "kernels.cuh"
#include "driver.cuh"
#include "tc_gemm.cuh"
#include "profile.cuh"
#include "rowsolve.cuh"

#include <algorithm>
#include <mutex>
#include <unordered_map>
#include <vector>

namespace lub {

lu_status check_device() {
  static int checked_dev = -1;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return LU_ERR_NO_DEVICE;
  if (dev == checked_dev) return LU_SUCCESS;
  int major = 0;
  if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev) !=
      cudaSuccess)
    return LU_ERR_NO_DEVICE;
  if (major != 10) return LU_ERR_NO_DEVICE;
  checked_dev = dev;
  return LU_SUCCESS;
}

static bool is_tc(lu_compute c) {
  return c == LU_COMPUTE_TC32 || c == LU_COMPUTE_TC32_BF16 ||
         c == LU_COMPUTE_TC32_E4M3 || c == LU_COMPUTE_TC32_SPLIT;
}

static TcOperand tc_kind(lu_compute c) {
  return c == LU_COMPUTE_TC32_BF16 ? TcOperand::BF16
       : c == LU_COMPUTE_TC32_E4M3 ? TcOperand::E4M3
       : c == LU_COMPUTE_TC32_SPLIT ? TcOperand::SPLIT16
                                    : TcOperand::F16;
}

// Workspace for the low-precision operand copies of an M x K by K x N
// tensor-core update: A (row-major, ld K), B (column-major, ld K), the e4m3
// scales of both and a scratch array for the per-tile maxima.
struct TcWs {
  size_t off_a = 0, off_b = 0, off_sa = 0, off_sb = 0, off_tmp = 0, bytes = 0;
};

static TcWs tc_ws_layout(size_t base, int64_t M, int64_t N, int64_t K,
                         TcOperand kind) {
  TcWs w;
  const size_t es = (size_t)tc_operand_bytes(kind);
  const int64_t ldk = tc_packed_k(kind, K);
  size_t off = align_up(base, 1024);
  w.off_a = off;  off = align_up(off + (size_t)M * ldk * es, 1024);
  w.off_b = off;  off = align_up(off + (size_t)N * ldk * es, 1024);
  const size_t ts = (size_t)(std::max(ceil_div(M, 128), ceil_div(N, 128)) + 1) * sizeof(int);
  w.off_sa = off;  off = align_up(off + ts, 256);
  w.off_sb = off;  off = align_up(off + ts, 256);
  w.off_tmp = off; off = align_up(off + ts, 256);
  w.bytes = off - base;
  return w;
}

// Pack A (M x K, column-major fp32, lda) into the row-major low-precision
// copy and B (K x N, column-major fp32, ldb) into the column-major copy,
// with per-tile scales for e4m3.
static lu_status tc_pack(cudaStream_t st, TcOperand kind, int64_t M, int64_t N,
                         int64_t K, const float* a, int64_t lda, const float* b,
                         int64_t ldb, char* ws, const TcWs& w) {
  const int64_t ldk = tc_packed_k(kind, K);
  int* sa = nullptr;
  int* sb = nullptr;
  ProfScope ps("pack_operands", st,
               (double)(M + N) * (4.0 * K + (double)tc_operand_bytes(kind) * ldk));
  if (tc_scaled(kind)) {
    sa = reinterpret_cast<int*>(ws + w.off_sa);
    sb = reinterpret_cast<int*>(ws + w.off_sb);
    int* tmp = reinterpret_cast<int*>(ws + w.off_tmp);
    LUB_TRY(launch_scale_rowtiles(st, M, K, a, lda, sa, tmp, tc_scale_bound(kind)));
    LUB_TRY(launch_scale_coltiles(st, K, N, b, ldb, sb, tmp, tc_scale_bound(kind)));
  }
  LUB_TRY(launch_pack_a(st, kind, M, K, a, lda, ws + w.off_a, ldk, sa));
  LUB_TRY(launch_pack_b(st, kind, K, N, b, ldb, ws + w.off_b, ldk, sb));
  return LU_SUCCESS;
}

// Rows [r0, r1) of the L21 copy and columns [c0, c1) of the U12 copy only,
// at their places in the packed buffers (for kinds with tile scales r0 and
// c0 are multiples of 128, so the ranges cover whole scale tiles of the
// full copies and their scales land in the same slots).
static lu_status tc_pack_range(cudaStream_t st, TcOperand kind, int64_t r0, int64_t r1,
                               int64_t c0, int64_t c1, int64_t K, const float* a,
                               int64_t lda, const float* b, int64_t ldb, char* ws,
                               const TcWs& w) {
  const bool scaled = tc_scaled(kind);
  if (scaled && (r0 % 128 != 0 || c0 % 128 != 0)) return LU_ERR_UNSUPPORTED;
  const int64_t ldk = tc_packed_k(kind, K);
  const int64_t es = tc_operand_bytes(kind);
  ProfScope ps("pack_operands", st,
               (double)((r1 - r0) + (c1 - c0)) * (4.0 * K + (double)es * ldk));
  int* tmp = reinterpret_cast<int*>(ws + w.off_tmp);
  if (r1 > r0) {
    int* sa = scaled ? reinterpret_cast<int*>(ws + w.off_sa) + r0 / 128 : nullptr;
    if (scaled)
      LUB_TRY(launch_scale_rowtiles(st, r1 - r0, K, a + r0, lda, sa, tmp, tc_scale_bound(kind)));
    LUB_TRY(launch_pack_a(st, kind, r1 - r0, K, a + r0, lda, ws + w.off_a + r0 * ldk * es,
                          ldk, sa));
  }
  if (c1 > c0) {
    int* sb = scaled ? reinterpret_cast<int*>(ws + w.off_sb) + c0 / 128 : nullptr;
    if (scaled)
      LUB_TRY(launch_scale_coltiles(st, K, c1 - c0, b + c0 * ldb, ldb, sb, tmp,
                                    tc_scale_bound(kind)));
    LUB_TRY(launch_pack_b(st, kind, K, c1 - c0, b + c0 * ldb, ldb,
                          ws + w.off_b + c0 * ldk * es, ldk, sb));
  }
  return LU_SUCCESS;
}

// C[M x N] -= Ap[r0 .., :] * Bp[:, c0 ..] from packed operands (r0, c0 are
// row / column offsets into the packed copies; multiples of 128 when the
// copies carry e4m3 tile scales).
static lu_status tc_apply(cudaStream_t st, TcOperand kind, int64_t M, int64_t N,
                          int64_t K, int64_t r0, int64_t c0, float* c,
                          int64_t ldc, char* ws, const TcWs& w, int* err,
                          int tiles_per_cta, int max_ctas = 0) {
  if (M <= 0 || N <= 0) return LU_SUCCESS;
  const int64_t ldk = tc_packed_k(kind, K);
  const int64_t es = tc_operand_bytes(kind);
  const int* sa = nullptr;
  const int* sb = nullptr;
  if (tc_scaled(kind)) {
    if (r0 % 128 != 0 || c0 % 128 != 0) return LU_ERR_INVALID_ARG;
    sa = reinterpret_cast<const int*>(ws + w.off_sa) + r0 / 128;
    sb = reinterpret_cast<const int*>(ws + w.off_sb) + c0 / 128;
  }
  // the split product runs over the three concatenated K segments
  const int64_t kk = kind == TcOperand::SPLIT16 ? ldk : K;
  // algorithmic bytes: C read + written once (fp32), both operands read once
  ProfScope ps("tc_update", st, 8.0 * M * N + (double)es * (M + N) * kk,
               2.0 * M * N * kk);
  return launch_tc_update(st, kind, M, N, kk, -1.0f, ws + w.off_a + r0 * ldk * es,
                          ldk, ws + w.off_b + c0 * ldk * es, ldk, c, ldc, sa, sb,
                          err, max_ctas, tiles_per_cta);
}

// C (fp32) -= A * B through the tensor cores (pack, then update).
static lu_status tc_update_fp32(cudaStream_t st, TcOperand kind, int64_t M,
                                int64_t N, int64_t K, float alpha,
                                const float* a, int64_t lda, const float* b,
                                int64_t ldb, float* c, int64_t ldc, char* ws,
                                const TcWs& w, int* err) {
  LUB_TRY(tc_pack(st, kind, M, N, K, a, lda, b, ldb, ws, w));
  if (alpha == -1.0f) return tc_apply(st, kind, M, N, K, 0, 0, c, ldc, ws, w, err, 0);
  const int64_t ldk = tc_packed_k(kind, K);
  const int* sa = tc_scaled(kind) ? reinterpret_cast<const int*>(ws + w.off_sa) : nullptr;
  const int* sb = tc_scaled(kind) ? reinterpret_cast<const int*>(ws + w.off_sb) : nullptr;
  return launch_tc_update(st, kind, M, N, kind == TcOperand::SPLIT16 ? ldk : K, alpha,
                          ws + w.off_a, ldk, ws + w.off_b, ldk, c, ldc, sa, sb, err);
}

// Internal streams of one device: panel work runs at the highest priority,
// the bulk of each trailing update at the lowest, ordered by two events.
constexpr int kMaxChunks = 16;  // column chunks of the host-memory entry
constexpr int kMaxBulkSteps = 8;  // outer steps per bulk pass (bulk_steps)

struct DevStreams {
  cudaStream_t panel = nullptr, update = nullptr, copy = nullptr, side = nullptr;
  cudaStream_t copy_out = nullptr;  // device-to-host, concurrent with `copy`
  cudaStream_t catchup = nullptr;   // the host entry's catch_up of arrived chunks
  cudaStream_t catchup_bulk = nullptr;  // its bulk updates (look-ahead)
  cudaStream_t catchup_early = nullptr;  // left-looking catch-up: early partial products
  cudaStream_t catchup_chain = nullptr;  // left-looking catch-up: the chain of block rows
  cudaEvent_t cu_done = nullptr;
  cudaEvent_t cu_packed = nullptr, cu_u2[2] = {nullptr, nullptr}, cu_join = nullptr;
  cudaEvent_t cu_out = nullptr;  // a chunk's catch-up done: its rows above it can go out
  // left-looking catch-up: a block row's solved rows are packed (cu_xp);
  // the early partial products of the block row of each parity are done
  cudaEvent_t cu_xp = nullptr, cu_early[2] = {nullptr, nullptr};
  // per outer step of the host entry: the step's block column is final
  // once what was queued on the panel (p) and side (s) streams has run
  std::vector<cudaEvent_t> step_p, step_s;
  cudaEvent_t chunk_in[kMaxChunks] = {};
  cudaEvent_t chunk_top[kMaxChunks] = {};  // the rows above a chunk's first column are in
  cudaEvent_t out_done = nullptr;
  cudaEvent_t diag_done = nullptr, small_done = nullptr, big_done = nullptr;
  cudaEvent_t diag1_done = nullptr;
  cudaEvent_t u1_done = nullptr, join_s = nullptr, spack_done = nullptr;
  cudaEvent_t copied = nullptr;
  cudaEvent_t fork = nullptr, join_p = nullptr, join_u = nullptr;
  cudaEvent_t packed = nullptr, updated = nullptr;
  cudaEvent_t done_with[kMaxBulkSteps + 2] = {};  // U2 done reading buffer b
  // left-looking look-ahead: the previous block is queued (ll_ready); the
  // early partial products of the block of each parity are done (ll_early)
  cudaEvent_t ll_ready = nullptr, ll_early[2] = {nullptr, nullptr};
};

static lu_status dev_streams(DevStreams** out) {
  static std::mutex mu;
  static std::unordered_map<int, DevStreams> cache;
  int dev = 0;
  LUB_CUDA_TRY(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(mu);
  auto it = cache.find(dev);
  if (it == cache.end()) {
    DevStreams d;
    int least = 0, greatest = 0;
    LUB_CUDA_TRY(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    LUB_CUDA_TRY(cudaStreamCreateWithPriority(&d.panel, cudaStreamNonBlocking, greatest));
    LUB_CUDA_TRY(cudaStreamCreateWithPriority(&d.update, cudaStreamNonBlocking, least));
    LUB_CUDA_TRY(cudaStreamCreateWithFlags(&d.copy, cudaStreamNonBlocking));
    LUB_CUDA_TRY(cudaStreamCreateWithFlags(&d.copy_out, cudaStreamNonBlocking));
    for (int q = 0; q < kMaxChunks; ++q) {
      LUB_CUDA_TRY(cudaEventCreateWithFlags(&d.chunk_in[q], cudaEventDisableTiming));
      LUB_CUDA_TRY(cudaEventCreateWithFlags(&d.chunk_top[q], cudaEventDisableTiming));
    }
    LUB_CUDA_TRY(cudaEventCreateWithFlags(&d.out_done, cudaEventDisableTiming));
    LUB_CUDA_TRY(cudaStreamCreateWithPriority(&d.catchup, cudaStreamNonBlocking, least));
    LUB_CUDA_TRY(cudaStreamCreateWithPriority(&d.catchup_bulk, cudaStreamNonBlocking, least));
    LUB_CUDA_TRY(cudaStreamCreateWithPriority(&d.catchup_early, cudaStreamNonBlocking, greatest));
    LUB_CUDA_TRY(cudaStreamCreateWithPriority(&d.catchup_chain, cudaStreamNonBlocking, greatest));
    LUB_CUDA_TRY(cudaEventCreateWithFlags(&d.cu_done, cudaEventDisableTiming));
    for (cudaEvent_t* e : {&d.cu_packed, &d.cu_u2[0], &d.cu_u2[1], &d.cu_join, &d.cu_out,
                           &d.cu_xp, &d.cu_early[0], &d.cu_early[1]})
      LUB_CUDA_TRY(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    LUB_CUDA_TRY(cudaStreamCreateWithPriority(&d.side, cudaStreamNonBlocking, greatest));
    for (cudaEvent_t* e : {&d.fork, &d.join_p, &d.join_u, &d.packed, &d.updated,
                           &d.copied,
                           &d.diag_done, &d.small_done, &d.big_done, &d.diag1_done,
                           &d.u1_done, &d.join_s,
                           &d.spack_done, &d.ll_ready, &d.ll_early[0], &d.ll_early[1]})
      LUB_CUDA_TRY(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    for (cudaEvent_t& e : d.done_with)
      LUB_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    it = cache.emplace(dev, d).first;
  }
  *out = &it->second;
  return LU_SUCCESS;
}

// At least `steps` per-step events in S (created on first need).
static lu_status step_events(DevStreams* S, int64_t steps) {
  static std::mutex mu;
  std::lock_guard<std::mutex> lk(mu);
  while ((int64_t)S->step_p.size() < steps) {
    cudaEvent_t e1 = nullptr, e2 = nullptr;
    LUB_CUDA_TRY(cudaEventCreateWithFlags(&e1, cudaEventDisableTiming));
    LUB_CUDA_TRY(cudaEventCreateWithFlags(&e2, cudaEventDisableTiming));
    S->step_p.push_back(e1);
    S->step_s.push_back(e2);
  }
  return LU_SUCCESS;
}

// Work queued on the side stream after this point follows what st has
// queued so far; join_side makes st wait for it.
static lu_status fork_side(cudaStream_t st, DevStreams* S) {
  LUB_CUDA_TRY(cudaEventRecord(S->fork, st));
  LUB_CUDA_TRY(cudaStreamWaitEvent(S->side, S->fork, 0));
  return LU_SUCCESS;
}
static lu_status join_side(cudaStream_t st, DevStreams* S) {
  LUB_CUDA_TRY(cudaEventRecord(S->join_s, S->side));
  LUB_CUDA_TRY(cudaStreamWaitEvent(st, S->join_s, 0));
  return LU_SUCCESS;
}

// Left-looking tensor-core updates have N = nb (block column) or M = nb
// (block row) and K = ofs: at most 2 n / 128 tiles, long in K, so they are
// split along K (up to kLlSplitMax ways) to fill the SMs.  With look-ahead
// the K range [0, ofs - nb) of a block's two updates is computed while the
// previous block is factored, and the previous block's own K = nb product
// after it: kLlSplitMax + 1 slabs per update, for blocks of either parity.
constexpr int kLlSplitMax = 4;
static size_t ll_part_layout(Plan* p, size_t off) {
  const int64_t n = p->n, nb = p->nb;
  const int64_t slab = std::max(((n + 3) / 4 * 4) * nb, ((nb + 3) / 4 * 4) * n);
  off = align_up(off, 1024);
  p->off_part = off;
  // per region: the early splits and the late (previous block's) product
  p->part_bytes = align_up((size_t)(kLlSplitMax + 1) * slab * 4, 1024);
  // regions: block parity x (block column, block row)
  return off + 4 * p->part_bytes;
}

// Outer steps whose bulk trailing updates share one pass by default: the
// pass then has K = 6 nb = 1536 (AI 384 flop/B of C traffic).  B200, TC32,
// nb = 256: n = 16384 273 / 275 / 272 TF/s and n = 32768 490 / 516 / 512
// TF/s with 4 / 6 / 8 steps per pass.
constexpr int kBulkSteps = 6;

lu_status make_plan(const lu_opts& o, int64_t m, int64_t n, lu_dtype dtype,
                    Plan* p) {
  if (m != n) return LU_ERR_UNSUPPORTED;
  if (n < 0) return LU_ERR_INVALID_ARG;
  if (o.ib != 8) return LU_ERR_UNSUPPORTED;
  if (o.nb < 8 || o.nb % 8 != 0 || o.nb > 4096) return LU_ERR_INVALID_ARG;
  const int dw = o.diag_width == 0 ? 128 : o.diag_width;
  if (dw < 8 || dw > 128 || dw % 8 != 0) return LU_ERR_INVALID_ARG;
  if (dtype != LU_F32 && dtype != LU_F16) return LU_ERR_UNSUPPORTED;
  if (o.variant != LU_RIGHT_LOOKING && o.variant != LU_LEFT_LOOKING)
    return LU_ERR_INVALID_ARG;
  // fp16 storage: the left-looking variant with fp16 tensor-core updates;
  // TC16 and FP16 (fp16 accumulation in the reference) run as TC32 with one
  // rounding of the fp32 sum to fp16
  lu_compute outer = (lu_compute)o.outer_update;
  if (dtype == LU_F16) {
    if (o.variant != LU_LEFT_LOOKING) return LU_ERR_UNSUPPORTED;
    if (outer == LU_COMPUTE_TC16 || outer == LU_COMPUTE_FP16) outer = LU_COMPUTE_TC32;
    if (outer != LU_COMPUTE_TC32) return LU_ERR_UNSUPPORTED;
  }
  // inner (rank-8 and within-block) updates always run in fp32, at least as
  // accurate as the reference's TC32 (any storage) or FP16 / TC16 (fp16
  // storage) inner updates
  const lu_compute inner = (lu_compute)o.inner_update;
  if (!(inner == LU_COMPUTE_FP32 || inner == LU_COMPUTE_TC32 ||
        (dtype == LU_F16 && (inner == LU_COMPUTE_FP16 || inner == LU_COMPUTE_TC16))))
    return LU_ERR_UNSUPPORTED;
  if (outer != LU_COMPUTE_FP32 && !is_tc(outer)) return LU_ERR_UNSUPPORTED;
  if (o.variant == LU_LEFT_LOOKING) {
    // e4m3 tile scales would have to follow the growing K range of the
    // left-looking products
    if (outer == LU_COMPUTE_TC32_E4M3 || outer == LU_COMPUTE_TC32_SPLIT)
      return LU_ERR_UNSUPPORTED;
  }
  p->n = n;
  p->nb = o.nb;
  p->diag_w = (int)std::min<int64_t>(dw, o.nb);
  p->inner = LU_COMPUTE_FP32;
  p->outer = outer;
  p->panel_fp32 = dtype == LU_F16 && o.variant == LU_LEFT_LOOKING && o.panel_fp32 != 0;
  p->variant = (lu_variant)o.variant;
  p->lookahead = o.lookahead != 0;
  p->dtype = dtype;
  size_t off = 0;
  p->off_status = off;  // [0] first bad pivot, [1] device wait error
  off += 256;
  if (p->variant == LU_LEFT_LOOKING && dtype == LU_F16) {
    p->diag_w = (int)std::min<int64_t>(p->nb, kLlSub);
    const int64_t ldk = (n + 15) / 16 * 16;
    p->ld_shadow = std::max<int64_t>(4, (n + 3) / 4 * 4);
    off = align_up(off, 1024);
    p->off_shadow = off;
    off = align_up(off + (size_t)p->ld_shadow * n * 4, 1024);
    p->off_lcopy = off;
    off = align_up(off + (size_t)n * ldk * 2, 1024);
    off = ll_part_layout(p, off);
    p->ws_bytes = off;
    return LU_SUCCESS;
  }
  if (p->variant == LU_LEFT_LOOKING) {
    p->diag_w = (int)std::min<int64_t>(p->nb, kLlSub);
    if (is_tc(p->outer) && n > p->nb) {
      // low-precision copies of all factored L columns (row-major) and U
      // rows (column-major), leading dimension round16(n)
      const int64_t ldk = (n + 15) / 16 * 16;
      const size_t es = (size_t)tc_operand_bytes(tc_kind(p->outer));
      off = align_up(off, 1024);
      p->off_lcopy = off;
      off = align_up(off + (size_t)n * ldk * es, 1024);
      p->off_ucopy = off;
      off = align_up(off + (size_t)n * ldk * es, 1024);
      off = ll_part_layout(p, off);
    }
    p->ws_bytes = off;
    return LU_SUCCESS;
  }
  // several outer steps per bulk pass (look-ahead, unscaled fp16 / bf16
  // operands): bulk_steps 0 (default: kBulkSteps) or 2..kMaxBulkSteps; 1
  // keeps one pass per step
  if (o.bulk_steps < 0 || o.bulk_steps > kMaxBulkSteps) return LU_ERR_INVALID_ARG;
  const bool grouping = is_tc(p->outer) && !tc_scaled(tc_kind(p->outer)) && p->lookahead;
  p->bulk_group = grouping ? (o.bulk_steps == 0 ? kBulkSteps : o.bulk_steps) : 1;
  p->bulk_pair = p->bulk_group >= 2;
  if (is_tc(p->outer) && n > p->nb) {
    // three operand buffers: with look-ahead the panel of step k writes its
    // copies while the bulk updates of steps k-1 and k-2 still read theirs;
    // q + 2 when q steps share a bulk pass (it reads the group's copies
    // until the panels of the next group's first two steps are done)
    const int64_t t = n - p->nb;
    TcWs w = tc_ws_layout(off, t, t, p->nb, tc_kind(p->outer));
    p->off_lcopy = w.off_a;
    off += (p->bulk_group >= 2 ? p->bulk_group + 2 : 3) * w.bytes;
  }
  p->ws_bytes = off;
  return LU_SUCCESS;
}

// Where a step's panel launches write the tensor-core operand copies of the
// rows / columns they finish (fp16 / bf16 kinds: no separate packing pass).
struct PackTarget {
  char* ws = nullptr;
  const TcWs* w = nullptr;
  int64_t ldk = 0, nb = 0;
  int bf16 = 0;
  // also the host entry's catch-up copy of the step's L columns (global
  // row r, column c at lp[r * ldl + c]); the step starts at column ofs
  char* lp = nullptr;
  int64_t ldl = 0, ofs = 0;
  // the launch of sub-block p0 (width wd) whose L rows / U columns start
  // offL / offU past the sub-block's edge
  LuPack at(int64_t p0, int wd, int64_t offL, int64_t offU) const {
    LuPack k;
    if (!ws) return k;
    k.pa = ws + w->off_a;
    k.pb = ws + w->off_b;
    k.ldk = ldk;
    k.row0 = p0 + wd + offL - nb;
    k.col0 = p0 + wd + offU - nb;
    k.k0 = (int)p0;
    k.bf16 = bf16;
    if (lp) {
      k.pa2 = lp;
      k.ldk2 = ldl;
      k.row02 = ofs + p0 + wd + offL;
      k.k02 = (int)(ofs + p0);
    }
    return k;
  }
};

static bool fused_pack(lu_compute outer) {
  return is_tc(outer) && !tc_scaled(tc_kind(outer));
}

static PackTarget pack_target(const Plan& p, char* ws, const TcWs& w) {
  PackTarget t;
  if (!fused_pack(p.outer)) return t;
  t.ws = ws;
  t.w = &w;
  t.ldk = tc_packed_k(tc_kind(p.outer), p.nb);
  t.nb = p.nb;
  t.bf16 = tc_kind(p.outer) == TcOperand::BF16;
  return t;
}

// Factor the outer block column/row starting at (ofs, ofs): width `in`,
// L rows [ofs, ofs + updm) and U columns [ofs, ofs + updc) (updc = updm for
// a whole factorization; fewer columns when only a column range is present).
static lu_status factor_block(const Plan& p, cudaStream_t st, float* a,
                              int64_t lda, int64_t ofs, int64_t in,
                              int64_t updm, int64_t updc, int* first_bad,
                              const PackTarget& pt = PackTarget()) {
  float* blk = a + ofs + ofs * lda;
  for (int64_t p0 = 0; p0 < in; p0 += p.diag_w) {
    const int w = (int)std::min<int64_t>(in - p0, p.diag_w);
    float* dg = blk + p0 + p0 * lda;
    {
      ProfScope ps("diag_factor", st, 8.0 * w * w, 2.0 * w * w * w / 3.0);
      LUB_TRY(launch_diag_factor(st, dg, lda, w, ofs + p0, first_bad));
    }
    const int64_t rest = updm - (p0 + w), restc = updc - (p0 + w);
    if (rest > 0 || restc > 0) {
      ProfScope ps("lupanel", st, 8.0 * (rest + restc) * w,
                   (double)(rest + restc) * (double)w * w);
      const LuPack pk = pt.at(p0, w, 0, 0);
      LUB_TRY(launch_lupanel(st, dg, lda, w, rest, restc, false, 0, 0, &pk));
    }
    if (p0 + w < in) {
      ProfScope ps("sgemm_chunk8", st, 0.0,
                   2.0 * w * ((double)(updm - p0 - w) * (in - p0 - w) +
                              (double)(in - p0 - w) * (updc - in)));
      // rest of the outer block column: rows [p0+w, updm), cols [p0+w, in);
      // rest of the outer block row: rows [p0+w, in), cols [in, updc)
      LUB_TRY(launch_sgemm_chunk8_2(
          st, updm - (p0 + w), in - (p0 + w), w, dg + w, lda, dg + (int64_t)w * lda,
          lda, dg + w + (int64_t)w * lda, lda,
          updc > in ? in - (p0 + w) : 0, updc - in, w, dg + w, lda,
          blk + p0 + in * lda, lda, blk + (p0 + w) + in * lda, lda));
    }
  }
  return LU_SUCCESS;
}

// The same factorization of the outer block for the look-ahead schedule,
// when it holds exactly two diagonal sub-blocks (in == 2 w): after the
// first diagonal block, only what the second one needs stays on the panel
// stream st -- the first w L rows and U columns of the sub-panel and their
// rank-w update of the second diagonal block -- while the rest of the
// sub-panel and of its update run on the side stream ss and overlap the
// second diagonal factorization.  Every element receives the same
// operations in the same order as in factor_block.
static lu_status factor_block_split(const Plan& p, cudaStream_t st, DevStreams* S,
                                    float* a, int64_t lda, int64_t ofs, int64_t in,
                                    int64_t updm, int64_t updc, int* first_bad,
                                    const PackTarget& pt = PackTarget()) {
  const int w = p.diag_w;
  if (in != 2 * w || updm <= in)
    return factor_block(p, st, a, lda, ofs, in, updm, updc, first_bad, pt);
  cudaStream_t ss = S->side;
  float* blk = a + ofs + ofs * lda;
  const int64_t big = updm - 2 * w;   // L rows beyond the outer block
  const int64_t bigc = updc - 2 * w;  // U columns beyond the outer block
  {
    ProfScope ps("diag_factor", st, 8.0 * w * w, 2.0 * w * w * w / 3.0);
    LUB_TRY(launch_diag_factor(st, blk, lda, w, ofs, first_bad));
  }
  LUB_CUDA_TRY(cudaEventRecord(S->diag_done, st));
  {
    ProfScope ps("lupanel", st, 2.0 * 8.0 * w * w, 2.0 * 2 * w * (double)w * w);
    LUB_TRY(launch_lupanel(st, blk, lda, w, w, w, false, 0, 0));
  }
  LUB_CUDA_TRY(cudaEventRecord(S->small_done, st));
  // side stream: the rest of the first sub-panel and of its update
  LUB_CUDA_TRY(cudaStreamWaitEvent(ss, S->diag_done, 0));
  {
    ProfScope ps("lupanel", ss, 8.0 * (big + bigc) * w, (double)(big + bigc) * (double)w * w);
    const LuPack pk = pt.at(0, w, w, w);
    LUB_TRY(launch_lupanel(ss, blk, lda, w, big, bigc, false, w, w, &pk));
  }
  LUB_CUDA_TRY(cudaStreamWaitEvent(ss, S->small_done, 0));
  {
    ProfScope ps("sgemm_chunk8", ss, 0.0, 2.0 * w * (double)(big + bigc) * w);
    // rows [2w, updm) x columns [w, 2w), and rows [w, 2w) x columns [2w, updc)
    LUB_TRY(launch_sgemm_chunk8_2(ss, big, w, w, blk + 2 * w, lda, blk + (int64_t)w * lda, lda,
                                  blk + 2 * w + (int64_t)w * lda, lda, w, bigc, w, blk + w, lda,
                                  blk + 2 * (int64_t)w * lda, lda,
                                  blk + w + 2 * (int64_t)w * lda, lda));
  }
  LUB_CUDA_TRY(cudaEventRecord(S->big_done, ss));
  // panel stream: the second diagonal block as soon as its own update is in
  {
    ProfScope ps("sgemm_chunk8", st, 0.0, 2.0 * (double)w * w * w);
    LUB_TRY(launch_sgemm_chunk8_2(st, w, w, w, blk + w, lda, blk + (int64_t)w * lda, lda,
                                  blk + w + (int64_t)w * lda, lda, 0, 0, 0, nullptr, lda,
                                  nullptr, lda, nullptr, lda));
  }
  float* dg1 = blk + w + (int64_t)w * lda;
  {
    ProfScope ps("diag_factor", st, 8.0 * w * w, 2.0 * w * w * w / 3.0);
    LUB_TRY(launch_diag_factor(st, dg1, lda, w, ofs + w, first_bad));
  }
  LUB_CUDA_TRY(cudaStreamWaitEvent(st, S->big_done, 0));
  {
    ProfScope ps("lupanel", st, 8.0 * (big + bigc) * w, (double)(big + bigc) * (double)w * w);
    const LuPack pk = pt.at(w, w, 0, 0);
    LUB_TRY(launch_lupanel(st, dg1, lda, w, big, bigc, false, 0, 0, &pk));
  }
  return LU_SUCCESS;
}

// Trailing update of outer step (ofs) restricted to rows [r0, n) x columns
// [c0, c0 + ncols): the block at (ofst + r0, ofst + c0).
static lu_status outer_update(const Plan& p, cudaStream_t st, float* a,
                              int64_t lda, int64_t ofs, int64_t r0, int64_t rows,
                              int64_t c0, int64_t cols, char* ws, const TcWs& w,
                              int* err, int tiles_per_cta, int max_ctas = 0) {
  if (rows <= 0 || cols <= 0) return LU_SUCCESS;
  const int64_t nb = p.nb, ofst = ofs + nb;
  float* c = a + (ofst + r0) + (ofst + c0) * lda;
  if (is_tc(p.outer))
    return tc_apply(st, tc_kind(p.outer), rows, cols, nb, r0, c0, c, lda, ws, w,
                    err, tiles_per_cta, max_ctas);
  ProfScope ps("sgemm_update", st, 8.0 * rows * cols, 2.0 * rows * cols * (double)nb);
  return launch_sgemm_update(st, rows, cols, nb, -1.0f, a + (ofst + r0) + ofs * lda,
                             lda, a + ofs + (ofst + c0) * lda, lda, 1.0f, c, lda,
                             false);
}

// Tiles per CTA of the trailing updates under look-ahead: few, so SMs free
// up often and the high-priority panel kernels get them quickly (measured on
// B200 at n = 16384: 2 tiles 133 TF/s, 8 tiles 124, 16 tiles 122).
constexpr int kU2Tiles = 2;
// ... except the bulk update U2b when it is large: then it runs as
// persistent CTAs on part of the SMs, leaving the rest to the panel streams.  B200, nb = 256, threshold
// 2048 tiles of 128 x 256: n = 16384 165 -> 181 TF/s, n = 32768 238 -> 243,
// n = 8192 unchanged (below the threshold it keeps the 2-tile CTAs).  Not
// for the split-fp16 update: two MMAs per tile make it compute-heavy enough
// to want every SM (n = 32768: 150 ms with all SMs, 194 ms capped).
constexpr int64_t kU2bPersistTiles = 2048;

// Right-looking factorization of the steps whose outer block starts in
// [col_begin, col_end), restricted to the columns [0, col_end) (rows always
// run to n): col_begin = 0, col_end = n is the whole factorization; the
// host-memory entry factors one arrived column range at a time (after
// catch_up gave it the earlier steps).  Without look-ahead every outer step
// runs in order on the caller's stream.  With look-ahead the trailing
// update of step k is split into U1 (the next block column and block row,
// which the panel of step k+1 needs), U2a (the block column and row after
// that, which U1 of step k+1 updates next) and U2b (everything else).  The
// panel, the operand packing and U1 run on a high-priority stream, U2a and
// U2b on a low-priority one; U1 of step k+1 waits only for U2a of step k,
// so the bulk U2b of step k overlaps the panels of steps k+1 and k+2.  The
// packed operands are double-buffered: packing step k+2 waits until U2 of
// step k has finished reading the same buffer.  Every element still
// receives its updates in the same order, so results are identical either
// way.
// Where rl_factor sends each finished block column (host-memory entry):
// after a step's panel, the rows [col_begin, n) of its block column are
// final (the rows above col_begin were final after catch_up and have gone
// out already); they go to h (ldh) on the copy stream `out`.
struct ColumnSink {
  float* h = nullptr;
  int64_t ldh = 0;
  cudaStream_t out = nullptr;
  // the left-looking catch-up's fp16 / bf16 copy of the L columns [0,
  // lp_cols), written by the panels of the steps inside that range
  char* lp = nullptr;
  int64_t ldl = 0, lp_cols = 0;
};

static lu_status rl_factor(const Plan& p, cudaStream_t st, float* a,
                           int64_t lda, char* ws, int* first_bad, int* err,
                           int64_t col_begin = 0, int64_t col_end = -1,
                           const ColumnSink* sink = nullptr) {
  const int64_t n = p.n, nb = p.nb;
  if (col_end < 0) col_end = n;
  const bool tc = is_tc(p.outer);
  // q steps per bulk pass (the host entry's chunks too, restricted to their
  // columns)
  const int q = p.bulk_group;
  const int nbuf = q >= 2 ? q + 2 : 3;
  TcWs w2[kMaxBulkSteps + 2];
  if (tc && n > nb) {
    w2[0] = tc_ws_layout(256, n - nb, n - nb, nb, tc_kind(p.outer));
    const size_t shift = w2[0].bytes;
    for (int b = 1; b < nbuf; ++b) {
      w2[b] = w2[0];
      w2[b].off_a += b * shift; w2[b].off_b += b * shift; w2[b].off_sa += b * shift;
      w2[b].off_sb += b * shift; w2[b].off_tmp += b * shift;
    }
  }
  const bool fused = fused_pack(p.outer);
  const bool la = p.lookahead && n > 2 * nb &&
                  !(tc && tc_scaled(tc_kind(p.outer)) && nb % 128 != 0);
  if (!la) {
    for (int64_t ofs = col_begin; ofs < col_end; ofs += nb) {
      const int64_t in = std::min(n - ofs, nb);
      LUB_TRY(factor_block(p, st, a, lda, ofs, in, n - ofs, col_end - ofs, first_bad,
                           pack_target(p, ws, w2[0])));
      if (sink) {
        ProfScope ps("copy_d2h", st, 4.0 * (double)(n - col_begin) * in);
        LUB_CUDA_TRY(cudaMemcpy2DAsync(sink->h + col_begin + ofs * sink->ldh,
                                       (size_t)sink->ldh * 4, a + col_begin + ofs * lda,
                                       (size_t)lda * 4, (size_t)(n - col_begin) * 4,
                                       (size_t)in, cudaMemcpyDeviceToHost, st));
      }
      const int64_t tr = n - (ofs + nb), tcn = col_end - (ofs + nb);
      if (tr <= 0 || tcn <= 0) continue;
      if (tc && !fused)
        LUB_TRY(tc_pack(st, tc_kind(p.outer), tr, tcn, nb, a + (ofs + nb) + ofs * lda,
                        lda, a + ofs + (ofs + nb) * lda, lda, ws, w2[0]));
      LUB_TRY(outer_update(p, st, a, lda, ofs, 0, tr, 0, tcn, ws, w2[0], err, 0));
    }
    return LU_SUCCESS;
  }
  DevStreams* S = nullptr;
  LUB_TRY(dev_streams(&S));
  if (sink) LUB_TRY(step_events(S, ceil_div(n, nb)));
  cudaStream_t sp = S->panel, su = S->update;
  LUB_CUDA_TRY(cudaEventRecord(S->fork, st));
  LUB_CUDA_TRY(cudaStreamWaitEvent(sp, S->fork, 0));
  LUB_CUDA_TRY(cudaStreamWaitEvent(su, S->fork, 0));
  lu_status status = LU_SUCCESS;
  int64_t step = 0;
  auto ok = [&](cudaError_t e) {
    if (e != cudaSuccess && status == LU_SUCCESS) status = LU_ERR_CUDA;
    return status == LU_SUCCESS;
  };
  cudaStream_t ss = S->side;
  LUB_CUDA_TRY(cudaStreamWaitEvent(ss, S->fork, 0));
  const int w = p.diag_w;
  const TcOperand kind = tc_kind(p.outer);
  // A step takes the deep schedule when its outer block holds two diagonal
  // blocks and at least two of them remain beyond it, in rows and columns.
  auto deep_step = [&](int64_t o) {
    const int64_t in_ = std::min(n - o, nb), tr_ = n - (o + nb), tc_ = col_end - (o + nb);
    return o < col_end && in_ == 2 * w && tr_ >= 2 * w && tc_ >= 2 * w &&
           !(tc && tc_scaled(kind));
  };
  bool pre = false;       // this step's first diagonal block is already queued
  bool prev_deep = false; // the previous step ran the deep schedule
  // steps of the current group whose bulk (rows and columns beyond their
  // trailing origin + 3 nb) waits to be applied together with later steps'
  int ngrp = 0;
  int grp_buf[kMaxBulkSteps] = {};
  int64_t grp_step[kMaxBulkSteps] = {};
  const int64_t ldk = tc && n > nb ? tc_packed_k(kind, nb) : 0;
  const int64_t es = tc ? tc_operand_bytes(kind) : 0;
  // block column [ofs, ofs + in) is final once the panel work queued so far
  // on sp (and, with `side`, on ss) has run
  auto sink_column = [&](int64_t ofs, int64_t in, bool side) {
    const int64_t t = ofs / nb;
    cudaEvent_t ep = S->step_p[t], es = S->step_s[t];
    if (!ok(cudaEventRecord(ep, sp)) || !ok(cudaEventRecord(es, side ? ss : sp)) ||
        !ok(cudaStreamWaitEvent(sink->out, ep, 0)) || !ok(cudaStreamWaitEvent(sink->out, es, 0)))
      return false;
    ProfScope ps("copy_d2h", sink->out, 4.0 * (double)(n - col_begin) * in);
    return ok(cudaMemcpy2DAsync(sink->h + col_begin + ofs * sink->ldh, (size_t)sink->ldh * 4,
                                a + col_begin + ofs * lda, (size_t)lda * 4,
                                (size_t)(n - col_begin) * 4, (size_t)in,
                                cudaMemcpyDeviceToHost, sink->out));
  };
  for (int64_t ofs = col_begin; ofs < col_end && status == LU_SUCCESS; ofs += nb, ++step) {
    const int64_t in = std::min(n - ofs, nb);
    const int64_t updm = n - ofs, updc = col_end - ofs;
    const int64_t tr = n - (ofs + nb);        // trailing rows
    const int64_t tcn = col_end - (ofs + nb); // trailing columns
    const int buf = (int)(step % nbuf);
    const TcWs& wk = w2[buf];
    PackTarget pt = pack_target(p, ws, wk);
    if (pt.ws && sink && sink->lp && ofs + in <= sink->lp_cols) {
      pt.lp = sink->lp;
      pt.ldl = sink->ldl;
      pt.ofs = ofs;
    }
    // this step's panel writes operand buffer `buf`: the bulk update that
    // last read it (step k - nbuf's) must have finished
    if (tc && step >= nbuf && (!ok(cudaStreamWaitEvent(sp, S->done_with[buf], 0)) ||
                               !ok(cudaStreamWaitEvent(ss, S->done_with[buf], 0))))
      break;
    // the previous step's update of this block column / row ran partly on
    // the side stream: a deep step only touches the diagonal square on the
    // panel stream and everything else on the side stream after it, any
    // other step waits for the side stream first
    if (prev_deep && !deep_step(ofs) && !ok(cudaStreamWaitEvent(sp, S->u1_done, 0))) break;
    if (deep_step(ofs)) {
      // Deep schedule.  Panel stream sp: first diagonal block, the first w
      // L rows / U columns of its sub-panel and their update of the second
      // diagonal block, the second diagonal block, the first nb L rows / U
      // columns of the second sub-panel; then the nb x nb diagonal square of
      // the next outer block gets this step's update and its first w x w
      // block is factored at once.
      // Side stream ss: the rest of both sub-panels and of the first one's
      // update, the rest of the operand packing and of the next block
      // column / row update (U1).  Low-priority stream su: U2 as before.
      float* blk = a + ofs + ofs * lda;
      float* dg1 = blk + w + (int64_t)w * lda;
      const int64_t big = updm - 2 * w, bigc = updc - 2 * w;
      if (!pre) {
        ProfScope ps("diag_factor", sp, 8.0 * w * w, 2.0 * w * w * w / 3.0);
        if ((status = launch_diag_factor(sp, blk, lda, w, ofs, first_bad)) != LU_SUCCESS) break;
        if (!ok(cudaEventRecord(S->diag_done, sp))) break;
      }
      {
        ProfScope ps("lupanel", sp, 16.0 * w * w, 2.0 * (double)w * w * w);
        if ((status = launch_lupanel(sp, blk, lda, w, w, w, false, 0, 0)) != LU_SUCCESS) break;
      }
      if (!ok(cudaEventRecord(S->small_done, sp))) break;
      if (!ok(cudaStreamWaitEvent(ss, S->diag_done, 0))) break;
      {
        ProfScope ps("lupanel", ss, 8.0 * (big + bigc) * w, (double)(big + bigc) * w * w);
        const LuPack pk = pt.at(0, w, w, w);
        if ((status = launch_lupanel(ss, blk, lda, w, big, bigc, false, w, w, &pk)) !=
            LU_SUCCESS)
          break;
      }
      if (!ok(cudaStreamWaitEvent(ss, S->small_done, 0))) break;
      {
        ProfScope ps("sgemm_chunk8", ss, 0.0, 2.0 * (double)(big + bigc) * w * w);
        status = launch_sgemm_chunk8_2(ss, big, w, w, blk + 2 * w, lda, blk + (int64_t)w * lda,
                                       lda, blk + 2 * w + (int64_t)w * lda, lda, w, bigc, w,
                                       blk + w, lda, blk + 2 * (int64_t)w * lda, lda,
                                       blk + w + 2 * (int64_t)w * lda, lda);
        if (status != LU_SUCCESS) break;
      }
      if (!ok(cudaEventRecord(S->big_done, ss))) break;
      {
        ProfScope ps("sgemm_chunk8", sp, 0.0, 2.0 * (double)w * w * w);
        status = launch_sgemm_chunk8_2(sp, w, w, w, blk + w, lda, blk + (int64_t)w * lda, lda,
                                       dg1, lda, 0, 0, 0, nullptr, lda, nullptr, lda, nullptr,
                                       lda);
        if (status != LU_SUCCESS) break;
      }
      {
        ProfScope ps("diag_factor", sp, 8.0 * w * w, 2.0 * w * w * w / 3.0);
        if ((status = launch_diag_factor(sp, dg1, lda, w, ofs + w, first_bad)) != LU_SUCCESS)
          break;
      }
      if (!ok(cudaEventRecord(S->diag1_done, sp))) break;
      if (!ok(cudaStreamWaitEvent(sp, S->big_done, 0))) break;
      // the nb x nb diagonal square of the next outer block: its update by
      // this step stays on the panel stream, so the next step's panel never
      // waits for the side stream's share of U1.  That update reads the
      // first sq rows of L21 and columns of U12, so the second sub-panel's
      // share of them is eliminated here too; the side stream takes the rest.
      const int64_t sq = std::min(nb, tcn);
      const int64_t mh = std::min(sq, big), nh = std::min(sq, bigc);
      {
        ProfScope ps("lupanel", sp, 8.0 * (mh + nh) * w, (double)(mh + nh) * w * w);
        const LuPack pk = pt.at(w, w, 0, 0);
        if ((status = launch_lupanel(sp, dg1, lda, w, mh, nh, false, 0, 0, &pk)) != LU_SUCCESS)
          break;
      }
      if (!ok(cudaStreamWaitEvent(ss, S->diag1_done, 0))) break;
      {
        ProfScope ps("lupanel", ss, 8.0 * (big - mh + bigc - nh) * w,
                     (double)(big - mh + bigc - nh) * w * w);
        const LuPack pk = pt.at(w, w, mh, nh);
        if ((status = launch_lupanel(ss, dg1, lda, w, big - mh, bigc - nh, false, mh, nh,
                                     &pk)) != LU_SUCCESS)
          break;
      }
      if (sink && !sink_column(ofs, in, true)) break;
      // L21 rows / U12 columns relative to the trailing part (ofs + nb)
      const float* L21 = a + (ofs + nb) + ofs * lda;
      const float* U12 = a + ofs + (ofs + nb) * lda;
      if (tc && !fused) {
        if ((status = tc_pack_range(sp, kind, 0, sq, 0, sq, nb, L21, lda, U12, lda, ws, wk)) !=
            LU_SUCCESS)
          break;
      }
      // the rest of U1 on the side stream reads these packed rows / columns
      // (or, on the FP32 path, the second sub-panel's first L rows / U columns)
      if (!ok(cudaEventRecord(S->spack_done, sp))) break;
      if (step > 0 && !ok(cudaStreamWaitEvent(sp, S->updated, 0))) break;
      if ((status = outer_update(p, sp, a, lda, ofs, 0, sq, 0, sq, ws, wk, err, 1)) !=
          LU_SUCCESS)
        break;
      pre = deep_step(ofs + nb);
      if (pre) {
        ProfScope ps("diag_factor", sp, 8.0 * w * w, 2.0 * w * w * w / 3.0);
        float* nblk = a + (ofs + nb) + (ofs + nb) * lda;
        if ((status = launch_diag_factor(sp, nblk, lda, w, ofs + nb, first_bad)) != LU_SUCCESS)
          break;
        if (!ok(cudaEventRecord(S->diag_done, sp))) break;
      }
      // side stream: the rest of the packing and of U1
      if (tc && !fused) {
        if ((status = tc_pack_range(ss, kind, sq, tr, sq, tcn, nb, L21, lda, U12, lda, ws,
                                    wk)) != LU_SUCCESS)
          break;
      }
      if (!ok(cudaEventRecord(S->packed, ss))) break;
      if (!ok(cudaStreamWaitEvent(ss, S->spack_done, 0))) break;
      if (step > 0 && !ok(cudaStreamWaitEvent(ss, S->updated, 0))) break;
      // U1 minus the square: block column below it, block row right of it
      status = outer_update(p, ss, a, lda, ofs, sq, tr - sq, 0, sq, ws, wk, err, 1);
      if (status == LU_SUCCESS)
        status = outer_update(p, ss, a, lda, ofs, 0, sq, sq, tcn - sq, ws, wk, err, 1);
      if (status != LU_SUCCESS) break;
      if (!ok(cudaEventRecord(S->u1_done, ss))) break;
      prev_deep = true;
    } else {
      status = factor_block_split(p, sp, S, a, lda, ofs, in, updm, updc, first_bad, pt);
      if (status != LU_SUCCESS) break;
      // factor_block_split ends on sp after the side stream's share
      if (sink && !sink_column(ofs, in, false)) break;
      prev_deep = false;
      pre = false;
      if (tr <= 0 || tcn <= 0) continue;
      if (tc && !fused) {
        status = tc_pack(sp, kind, tr, tcn, nb, a + (ofs + nb) + ofs * lda, lda,
                         a + ofs + (ofs + nb) * lda, lda, ws, wk);
        if (status != LU_SUCCESS) break;
      }
      if (!ok(cudaEventRecord(S->packed, sp))) break;
      // U1 after U2a of the previous step (same elements, earlier step first)
      if (step > 0 && !ok(cudaStreamWaitEvent(sp, S->updated, 0))) break;
      const int64_t b = std::min(nb, tcn);
      status = outer_update(p, sp, a, lda, ofs, 0, tr, 0, b, ws, wk, err, 1);
      if (status == LU_SUCCESS && tcn > nb)
        status = outer_update(p, sp, a, lda, ofs, 0, std::min(nb, tr), nb, tcn - nb, ws, wk,
                              err, 1);
      if (status != LU_SUCCESS) break;
    }
    if (tr > nb && tcn > nb) {
      if (!ok(cudaStreamWaitEvent(su, S->packed, 0))) break;
      // U2a: block column and row k+2 (rows / columns [nb, 2nb) of the trailing part)
      const int64_t b2c = std::min(nb, tcn - nb), b2r = std::min(nb, tr - nb);
      status = outer_update(p, su, a, lda, ofs, nb, tr - nb, nb, b2c, ws, wk, err, kU2Tiles);
      if (status == LU_SUCCESS && tcn > 2 * nb)
        status = outer_update(p, su, a, lda, ofs, nb, b2r, 2 * nb, tcn - 2 * nb, ws, wk,
                              err, kU2Tiles);
      if (status != LU_SUCCESS) break;
      if (!ok(cudaEventRecord(S->updated, su))) break;
      // U2b: the rest.  Paired steps: the first of two defers all but the
      // first block row / column of its U2b, which the second step's U2b
      // covers exactly; that pass then applies both steps' products.
      if (tr > 2 * nb && tcn > 2 * nb) {
        const int64_t t2b = ceil_div(tr - 2 * nb, 128) * ceil_div(tcn - 2 * nb, 256);
        const bool persist = tc && tc_kind(p.outer) != TcOperand::SPLIT16 &&
                             t2b >= kU2bPersistTiles;
        const int tiles = persist ? 0 : kU2Tiles;
        // the bulk's share of the SMs (the rest for the panel streams): 2/3,
        // 3/4 from 4096 tiles, 7/8 from 8192 (B200, four steps per pass:
        // n = 16384 268 / 270 / 263 TF/s at 2/3, 3/4, 7/8 for its first
        // passes; n = 32768 478 / 484 / 492; all SMs: 220 and 430)
        const int share_num = t2b >= 4 * kU2bPersistTiles ? 7 : t2b >= 2 * kU2bPersistTiles ? 3 : 2;
        const int share_den = t2b >= 4 * kU2bPersistTiles ? 8 : t2b >= 2 * kU2bPersistTiles ? 4 : 3;
        const int ctas = persist ? std::max(1, sm_count() * share_num / share_den) : 0;
        // defer this step's bulk too while the group has room and the next
        // step has a bulk region of its own (one block smaller)
        const bool defer = q >= 2 && ngrp + 1 < q && tr > 3 * nb && tcn > 3 * nb;
        // rows [r0, r0 + rows) x columns [c0, c0 + cols) of this step's
        // trailing part -= the pending steps' products and this step's, in
        // one pass: step j's copy of this step's trailing row / column x
        // sits at x + (step - j) nb
        auto group_update = [&](int64_t r0, int64_t rows, int64_t c0, int64_t cols,
                                int tiles_, int ctas_) -> lu_status {
          if (rows <= 0 || cols <= 0) return LU_SUCCESS;
          int64_t ks[kMaxBulkSteps];
          const void* as[kMaxBulkSteps];
          const void* bs[kMaxBulkSteps];
          int ns = 0;
          for (int g = 0; g <= ngrp; ++g) {
            const bool own = g == ngrp;
            const TcWs& wg = w2[own ? buf : grp_buf[g]];
            const int64_t sh = own ? 0 : (step - grp_step[g]) * nb;
            ks[ns] = nb;
            as[ns] = ws + wg.off_a + (r0 + sh) * ldk * es;
            bs[ns] = ws + wg.off_b + (c0 + sh) * ldk * es;
            ++ns;
          }
          float* c = a + (ofs + nb + r0) + (ofs + nb + c0) * lda;
          ProfScope ps("tc_update", su, 8.0 * rows * cols + (double)es * (rows + cols) * nb * ns,
                       2.0 * rows * (double)cols * nb * ns);
          return launch_tc_update_sets(su, kind, rows, cols, ns, ks, as, bs, ldk, c, lda, err,
                                       ctas_, tiles_);
        };
        if (defer) {
          // the block row and column at 2 nb get every pending product now;
          // everything beyond waits for the group's pass
          status = group_update(2 * nb, nb, 2 * nb, tcn - 2 * nb, kU2Tiles, 0);
          if (status == LU_SUCCESS)
            status = group_update(3 * nb, tr - 3 * nb, 2 * nb, nb, kU2Tiles, 0);
          if (status != LU_SUCCESS) break;
          grp_buf[ngrp] = buf;
          grp_step[ngrp] = step;
          ++ngrp;
        } else if (ngrp > 0) {
          // the group's pass: rows / columns [2 nb, ...) of this step's
          // trailing part with all of the group's products
          status = group_update(2 * nb, tr - 2 * nb, 2 * nb, tcn - 2 * nb, tiles, ctas);
          if (status != LU_SUCCESS) break;
          for (int g = 0; g < ngrp; ++g)
            if (!ok(cudaEventRecord(S->done_with[grp_buf[g]], su))) break;
          if (status != LU_SUCCESS) break;
          ngrp = 0;
        } else {
          status = outer_update(p, su, a, lda, ofs, 2 * nb, tr - 2 * nb, 2 * nb,
                                tcn - 2 * nb, ws, wk, err, tiles, ctas);
          if (status != LU_SUCCESS) break;
        }
      }
      const bool pending = ngrp > 0 && grp_buf[ngrp - 1] == buf && grp_step[ngrp - 1] == step;
      if (!pending && !ok(cudaEventRecord(S->done_with[buf], su))) break;
    } else if (tr > 0 && tcn > 0) {
      cudaStream_t last = prev_deep ? ss : sp;
      if (!ok(cudaEventRecord(S->updated, last))) break;
      if (!ok(cudaEventRecord(S->done_with[buf], last))) break;
    }
  }
  // join (also on the error path, so the caller's stream stays ordered)
  cudaEventRecord(S->join_p, sp);
  cudaEventRecord(S->join_u, su);
  cudaEventRecord(S->join_s, S->side);
  cudaStreamWaitEvent(st, S->join_p, 0);
  cudaStreamWaitEvent(st, S->join_u, 0);
  cudaStreamWaitEvent(st, S->join_s, 0);
  return status;
}

// The U part of outer step ofs (block width in) for the columns [c0, c0 +
// nc) right of its block: the unit-lower solves with the block's diagonal
// sub-blocks and the rank-w update between them, exactly as factor_block
// applies them to a column right of the block.  With xp given, the solved
// rows also go to the fp16 / bf16 B operand xp (column j of the range at
// xp[j * ldx + ofs + i]).
static lu_status u_solve_cols(const Plan& p, cudaStream_t st, float* a, int64_t lda,
                              int64_t ofs, int64_t in, int64_t c0, int64_t nc,
                              void* xp = nullptr, int64_t ldx = 0, bool bf16 = false) {
  float* blk = a + ofs + ofs * lda;
  for (int64_t p0 = 0; p0 < in; p0 += p.diag_w) {
    const int dw = (int)std::min<int64_t>(in - p0, p.diag_w);
    float* dg = blk + p0 + p0 * lda;
    {
      ProfScope ps("lupanel", st, 8.0 * nc * dw, (double)nc * dw * dw);
      LuPack pk;
      pk.pb = xp;
      pk.ldk = ldx;
      pk.k0 = (int)(ofs + p0);
      pk.bf16 = bf16;
      LUB_TRY(launch_lupanel(st, dg, lda, dw, 0, nc, false, 0, c0 - (ofs + p0 + dw),
                             xp ? &pk : nullptr));
    }
    if (p0 + dw < in) {
      ProfScope ps("sgemm_chunk8", st, 0.0, 2.0 * dw * (double)(in - p0 - dw) * nc);
      LUB_TRY(launch_sgemm_chunk8_2(st, 0, 0, 0, nullptr, lda, nullptr, lda, nullptr, lda,
                                    in - (p0 + dw), nc, dw, dg + dw, lda,
                                    blk + p0 + (c0 - ofs) * lda, lda,
                                    blk + (p0 + dw) + (c0 - ofs) * lda, lda));
    }
  }
  return LU_SUCCESS;
}

// Give the columns [c0, c1) (all rows) the outer steps whose blocks start
// before c0, in step order: per step the U part of its panel -- the
// unit-lower solves with the outer block's diagonal sub-blocks and the
// rank-w update between them, exactly as factor_block applies them to a
// column right of the block -- then its trailing update.  Every element
// receives the same operations in the same order as when rl_factor runs
// over the whole matrix, so the factors are bit-identical.
// With S given, step t waits for S->step_p / step_s[t] first (the step's
// block column final), so the catch-up of an arrived chunk can run beside
// the factorization of the chunk before it; and the trailing update of
// step t is split into U1 (the next block row, rows [nb, 2 nb) of the
// trailing part, on st) and U2 (the rest, on S->catchup_bulk), so that U2
// of step t runs beside the solves and U1 of step t+1: the solves of step
// t need U1 of t-1 and U2 of t-2, U1 of step t needs U2 of t-1 (per-parity
// events), and U2 runs in step order on its own stream.  The operands of
// step t go to buffer t % 2 of wk: packing step t+2 follows U1 of step
// t+1, which follows U2 of step t, the last reader of that buffer.
static lu_status catch_up(const Plan& p, cudaStream_t st, float* a, int64_t lda, char* ws,
                          const TcWs* wk, int* err, int64_t c0, int64_t c1,
                          DevStreams* S = nullptr) {
  const int64_t n = p.n, nb = p.nb, nc = c1 - c0;
  const bool tc = is_tc(p.outer);
  const TcOperand kind = tc_kind(p.outer);
  cudaStream_t sb = S ? S->catchup_bulk : nullptr;
  if (S) {
    LUB_CUDA_TRY(cudaEventRecord(S->cu_join, st));
    LUB_CUDA_TRY(cudaStreamWaitEvent(sb, S->cu_join, 0));
  }
  // Two steps per bulk pass (look-ahead, unscaled operands): an even step
  // updates only the block row below its U1 (U2a) and leaves the rest to the
  // next step, whose U2 region is exactly that rest; the odd step's pass
  // then applies both steps' products (C - (L_t U_t + L_t+1 U_t+1)).  Both
  // operand buffers stay in use until that pass, whose completion releases
  // them (cu_u2 of both parities).
  const int64_t nsteps = ceil_div(c0, nb);
  const bool pairing = S && tc && p.bulk_pair && !tc_scaled(kind);
  bool deferred = false;
  for (int64_t ofs = 0; ofs < c0; ofs += nb) {
    const int64_t t = ofs / nb;
    const TcWs& w = wk[S ? t % 2 : 0];
    if (S) {
      LUB_CUDA_TRY(cudaStreamWaitEvent(st, S->step_p[t], 0));
      LUB_CUDA_TRY(cudaStreamWaitEvent(st, S->step_s[t], 0));
      if (t >= 2) LUB_CUDA_TRY(cudaStreamWaitEvent(st, S->cu_u2[t % 2], 0));
    }
    const int64_t in = std::min(n - ofs, nb);
    LUB_TRY(u_solve_cols(p, st, a, lda, ofs, in, c0, nc));
    const int64_t tr = n - (ofs + nb);
    if (tr <= 0) continue;
    const int64_t cr = c0 - (ofs + nb);  // column offset in the trailing part
    if (tc)
      LUB_TRY(tc_pack_range(st, kind, 0, tr, cr, cr + nc, nb, a + (ofs + nb) + ofs * lda, lda,
                            a + ofs + (ofs + nb) * lda, lda, ws, w));
    if (!S) {
      LUB_TRY(outer_update(p, st, a, lda, ofs, 0, tr, cr, nc, ws, w, err, 0));
      continue;
    }
    const int64_t r1 = std::min(tr, nb);  // U1: rows [0, r1) of the trailing part
    bool u1_ordered = false;
    if (deferred) {
      // U1 of this step follows the previous step's U2a (its block row); the
      // event is about to be re-recorded for the pass below
      LUB_CUDA_TRY(cudaStreamWaitEvent(st, S->cu_u2[(t - 1) % 2], 0));
      u1_ordered = true;
      // rows [nb, tr) of this step = rows [2 nb, ...) of the previous step
      LUB_CUDA_TRY(cudaEventRecord(S->cu_packed, st));
      LUB_CUDA_TRY(cudaStreamWaitEvent(sb, S->cu_packed, 0));
      const TcWs& wp = wk[(t - 1) % 2];
      const int64_t ldk = tc_packed_k(kind, nb);
      const int64_t es = tc_operand_bytes(kind);
      const int64_t crp = cr + nb;  // the chunk's columns in the previous step's copy
      float* c = a + (ofs + nb + r1) + c0 * lda;
      ProfScope ps("tc_update", sb, 8.0 * (tr - r1) * nc + 2.0 * es * (tr - r1 + nc) * nb,
                   4.0 * (tr - r1) * (double)nc * nb);
      LUB_TRY(launch_tc_update2(sb, kind, tr - r1, nc, nb, ws + wp.off_a + 2 * nb * ldk * es,
                                ws + wp.off_b + crp * ldk * es, nb,
                                ws + w.off_a + r1 * ldk * es, ws + w.off_b + cr * ldk * es,
                                ldk, c, lda, err, 0, 0));
      LUB_CUDA_TRY(cudaEventRecord(S->cu_u2[(t - 1) % 2], sb));
      LUB_CUDA_TRY(cudaEventRecord(S->cu_u2[t % 2], sb));
      deferred = false;
    } else if (tr > r1) {
      // an even step whose next step still has a U2 region: update only the
      // block row below U1 now
      const bool defer = pairing && t % 2 == 0 && t + 1 < nsteps && tr > 2 * nb;
      const int64_t rows = defer ? nb : tr - r1;
      LUB_CUDA_TRY(cudaEventRecord(S->cu_packed, st));
      LUB_CUDA_TRY(cudaStreamWaitEvent(sb, S->cu_packed, 0));
      LUB_TRY(outer_update(p, sb, a, lda, ofs, r1, rows, cr, nc, ws, w, err, 0));
      LUB_CUDA_TRY(cudaEventRecord(S->cu_u2[t % 2], sb));
      deferred = defer;
    }
    if (t >= 1 && !u1_ordered) LUB_CUDA_TRY(cudaStreamWaitEvent(st, S->cu_u2[(t - 1) % 2], 0));
    LUB_TRY(outer_update(p, st, a, lda, ofs, 0, r1, cr, nc, ws, w, err, 0));
  }
  if (S) {
    LUB_CUDA_TRY(cudaEventRecord(S->cu_join, sb));
    LUB_CUDA_TRY(cudaStreamWaitEvent(st, S->cu_join, 0));
  }
  return LU_SUCCESS;
}

// Operands of the left-looking catch-up (catch_up_ll), kept across the
// chunks of one host-entry call: the L columns of every outer step left of
// the last chunk as tensor-core A rows (lp, row stride ldl elements, column
// k of L at element k), the solved U rows of the current chunk as B
// columns (xp, stride ldx), and the split-K slabs of its block-row updates.
struct LlCatchup {
  char* lp = nullptr;
  int64_t ldl = 0;
  char* xp = nullptr;
  int64_t ldx = 0;
  float* part = nullptr;  // two sets of kLlCatchupSplitMax slabs of `slab` floats
  int64_t slab = 0;
  int ksplit_max = 1;
};
constexpr int kLlCatchupSplitMax = 8;
// outer steps per pass over the chunk's rows below c0, and per copy out
constexpr int kLlCatchupGroup = 8;
// column chunks of the host entry with the left-looking catch-up
constexpr int kLlChunks = 8;

// One block row of the left-looking catch-up, on a block whose diagonal
// block (in x in, factored) sits at blk (leading dimension lda) and whose
// block row (in x nc, the earlier products but the last one subtracted)
// starts coff columns right of it: R -= La Xb (K = kl; kl = 0: nothing to
// subtract), then the unit-lower solve in place, its fp16 / bf16 copy to xo
// (column q, row i at xo[q * ldx + i]).  fused: one ll_rowsolve launch;
// otherwise the tensor-core update and the blocked U-panel solves (diag_w
// rows at a time, rank-8 updates between them) -- the same solve, bit for
// bit.
lu_status catchup_row_step(cudaStream_t st, bool fused, bool bf16, float* blk, int64_t lda,
                           int64_t in, int64_t coff, int64_t nc, int64_t kl, const void* la,
                           int64_t lda_k, const void* xb, void* xo, int64_t ldx, int diag_w,
                           int* err, const EarlyPart& ep) {
  const TcOperand kind = bf16 ? TcOperand::BF16 : TcOperand::F16;
  float* rows = blk + coff * lda;
  const int64_t es = tc_operand_bytes(kind);
  if (fused) {
    ProfScope ps("rowsolve", st, 8.0 * in * nc + 2.0 * in * in + es * (in + nc) * kl,
                 2.0 * in * (double)nc * kl + (double)in * in * nc);
    RowSolveArgs g;
    g.r = rows;
    g.ldr = lda;
    g.l = blk;
    g.ldl = lda;
    g.la = la;
    g.lda_k = lda_k;
    g.xb = xb;
    g.xo = xo;
    g.ldx = ldx;
    g.nc = nc;
    g.in = (int)in;
    g.kl = (int)kl;
    g.part = ep.part;
    g.ns = ep.ns;
    g.slab = ep.slab;
    g.ldp = ep.ldp;
    return launch_ll_rowsolve(st, bf16, g);
  }
  if (ep.ns > 0) {
    ProfScope ps("splitk_finish", st, 4.0 * (ep.ns + 2) * (double)in * nc);
    LUB_TRY(launch_splitk_finish(st, in, nc, ep.ns, ep.part, -1.0f, rows, false, lda, nullptr,
                                 0));
  }
  if (kl > 0) {
    ProfScope ps("tc_update", st, 8.0 * in * nc + (double)es * (in + nc) * kl,
                 2.0 * in * (double)nc * kl);
    LUB_TRY(launch_tc_update(st, kind, in, nc, kl, -1.0f, la, lda_k, xb, ldx, rows, lda,
                             nullptr, nullptr, err));
  }
  Plan q;
  q.diag_w = diag_w;
  return u_solve_cols(q, st, blk, lda, 0, in, coff, nc, xo, ldx, bf16);
}

// The catch-up of the columns [c0, c1) in left-looking order (unscaled fp16 /
// bf16 operands, several outer steps per bulk pass): block row t of the
// chunk (rows [t nb, (t+1) nb)) first receives the products of all earlier
// steps (K = t nb), then the U part of step t (the unit-lower solve with
// its diagonal block), which also writes the solved rows as the B operand of
// the later block rows.  The products with the solved rows of steps up to
// t-2 (the early part, K = (t-1) nb: split-K partial products in fixed
// slabs, summed in split order, so every run gives the same result) are
// computed and subtracted on S->catchup_early while block row t-1 is
// solved; only the last step's product (K = nb) stays on the chain of
// solves, fused with the solve into one launch (ll_rowsolve) where the
// block fits it.  The L columns of the earlier steps (A rows) come from the
// factorization's own panel kernels (ColumnSink::lp).  The rows [c0, n)
// receive L X in passes of kLlCatchupGroup steps on S->catchup_bulk as the solved
// rows come in (the chunk's rows [c0, n) may still be arriving when the
// chain starts: rows_in marks them in), and each group's solved rows go to
// the host at once on sink.out.  Against the step-by-step catch-up this
// saves the per-step passes over all rows below each block row (the chain
// of solves runs beside fewer, larger updates); the sums are rounded once
// per update instead of once per step, as in the grouped bulk passes of
// the factorization itself.
static lu_status catch_up_ll(const Plan& p, cudaStream_t st, float* a, int64_t lda,
                             LlCatchup* cu, int* err, int64_t c0, int64_t c1, DevStreams* S,
                             const ColumnSink& sink, cudaEvent_t rows_in) {
  const int64_t n = p.n, nb = p.nb, nc = c1 - c0;
  const TcOperand kind = tc_kind(p.outer);
  const int64_t es = tc_operand_bytes(kind);
  cudaStream_t sb = S->catchup_bulk, se = S->catchup_early;
  LUB_CUDA_TRY(cudaEventRecord(S->cu_join, st));
  LUB_CUDA_TRY(cudaStreamWaitEvent(sb, S->cu_join, 0));
  // the passes over the rows [c0, n) wait for them to arrive (rows_in); the
  // chain of block rows needs only the rows above c0
  LUB_CUDA_TRY(cudaStreamWaitEvent(sb, rows_in, 0));
  LUB_CUDA_TRY(cudaStreamWaitEvent(se, S->cu_join, 0));
  const int ctas = std::max(1, sm_count() * 3 / 4);
  const int64_t nsteps = ceil_div(c0, nb);
  // one fused launch per block row (late product + solve, and the sum of
  // its early partial products) where it fits
  const bool fused = rowsolve_supported(nb, nb, cu->ldx) && cu->ldl % 8 == 0;
  // The L columns of every earlier step are in lp already: the
  // factorization's panels wrote them with the step (its step events).
  // the partial products of block row r go to slab set r % 2
  std::vector<int> nslabs(nsteps, 0);
  const int64_t set_floats = (int64_t)cu->ksplit_max * cu->slab;
  int64_t k0 = 0;  // first row of the group whose bulk pass is pending
  for (int64_t t = 0; t < nsteps; ++t) {
    const int64_t ofs = t * nb, in = std::min(nb, c0 - ofs);
    LUB_CUDA_TRY(cudaStreamWaitEvent(st, S->step_p[t], 0));
    LUB_CUDA_TRY(cudaStreamWaitEvent(st, S->step_s[t], 0));
    // row t's products with the solved rows up to t-2 (on se, two
    // iterations ago)
    if (t >= 2) LUB_CUDA_TRY(cudaStreamWaitEvent(st, S->cu_early[t % 2], 0));
    const int64_t k_late = ofs - nb;
    EarlyPart ep;
    if (fused && nslabs[t] > 0) {
      ep.part = cu->part + (t % 2) * set_floats;
      ep.ns = nslabs[t];
      ep.slab = splitk_slab_floats(in, nc);
      ep.ldp = (in + 3) / 4 * 4;
    }
    LUB_TRY(catchup_row_step(st, fused, kind == TcOperand::BF16, a + ofs + ofs * lda, lda, in,
                             c0 - ofs, nc, t > 0 ? nb : 0,
                             t > 0 ? cu->lp + (ofs * cu->ldl + k_late) * es : nullptr, cu->ldl,
                             t > 0 ? cu->xp + k_late * es : nullptr, cu->xp + ofs * es,
                             cu->ldx, p.diag_w, err, ep));
    // on se: block row t+2's early part (K = (t+1) nb: the solved rows up to
    // this one) beside the solve of block row t+1; its slab set was last
    // read by the solve of block row t, just done
    LUB_CUDA_TRY(cudaEventRecord(S->cu_xp, st));
    LUB_CUDA_TRY(cudaStreamWaitEvent(se, S->cu_xp, 0));
    if (t + 2 < nsteps) {
      const int64_t o2 = ofs + 2 * nb, ke = ofs + nb;
      const int64_t in2 = std::min(nb, c0 - o2);
      const int64_t tiles = ceil_div(in2, 128) * ceil_div(nc, 256);
      const int ks = tc_split_choice(tiles, ke, (int)es, sm_count(), cu->ksplit_max);
      float* set = cu->part + (t % 2) * set_floats;
      int ns = 0;
      {
        ProfScope ps("tc_update", se, 4.0 * ks * in2 * nc + (double)es * (in2 + nc) * ke,
                     2.0 * in2 * (double)nc * ke);
        LUB_TRY(launch_tc_partials(se, kind, in2, nc, ke, cu->lp + o2 * cu->ldl * es, cu->ldl,
                                   cu->xp, cu->ldx, ks, set, 0, &ns, err));
      }
      nslabs[t + 2] = ns;
      if (!fused) {
        ProfScope ps("splitk_finish", se, 4.0 * (ns + 2) * (double)in2 * nc);
        LUB_TRY(launch_splitk_finish(se, in2, nc, ns, set, -1.0f, a + o2 + c0 * lda, false,
                                     lda, nullptr, 0));
      }
      LUB_CUDA_TRY(cudaEventRecord(S->cu_early[t % 2], se));
    }
    const int64_t k1 = ofs + in;
    if ((t + 1) % kLlCatchupGroup != 0 && t + 1 < nsteps) continue;
    LUB_CUDA_TRY(cudaEventRecord(S->cu_packed, st));
    LUB_CUDA_TRY(cudaStreamWaitEvent(sb, S->cu_packed, 0));
    if (n > c0) {
      ProfScope ps("tc_update", sb, 8.0 * (n - c0) * nc + (double)es * (n - c0 + nc) * (k1 - k0),
                   2.0 * (n - c0) * (double)nc * (k1 - k0));
      LUB_TRY(launch_tc_update(sb, kind, n - c0, nc, k1 - k0, -1.0f,
                               cu->lp + (c0 * cu->ldl + k0) * es, cu->ldl, cu->xp + k0 * es,
                               cu->ldx, a + c0 + c0 * lda, lda, nullptr, nullptr, err, ctas, 0));
    }
    // rows [k0, k1) of the chunk are final: out at once
    LUB_CUDA_TRY(cudaStreamWaitEvent(sink.out, S->cu_packed, 0));
    {
      ProfScope ps("copy_d2h", sink.out, 4.0 * (double)(k1 - k0) * nc);
      LUB_CUDA_TRY(cudaMemcpy2DAsync(sink.h + k0 + c0 * sink.ldh, (size_t)sink.ldh * 4,
                                     a + k0 + c0 * lda, (size_t)lda * 4, (size_t)(k1 - k0) * 4,
                                     (size_t)nc, cudaMemcpyDeviceToHost, sink.out));
    }
    k0 = k1;
  }
  LUB_CUDA_TRY(cudaEventRecord(S->cu_join, sb));
  LUB_CUDA_TRY(cudaStreamWaitEvent(st, S->cu_join, 0));
  LUB_CUDA_TRY(cudaEventRecord(S->cu_join, se));
  LUB_CUDA_TRY(cudaStreamWaitEvent(st, S->cu_join, 0));
  return LU_SUCCESS;
}

// K splits of a step's two concurrent left-looking updates (block column
// updm x in, block row in x (updm - in), K = ofs), chosen over their tiles
// together.
static int ll_split(int64_t updm, int64_t in, int64_t ofs, int64_t es) {
  const int64_t tiles = ceil_div(updm, 128) * ceil_div(in, 256) +
                        (updm > in ? ceil_div(in, 128) * ceil_div(updm - in, 256) : 0);
  return tc_split_choice(tiles, ofs, (int)es, sm_count(), kLlSplitMax);
}

// The inside of one left-looking outer block (columns [ofs, ofs + in) of an
// n x n matrix x, ld ldx, already updated by all columns left of ofs): the
// block is factored as sub-blocks of at most kLlSub columns; sub-block c
// first receives the FP32 update from the block's own columns [ofs, c)
// (its column below and its row to the right), then the Crout diagonal
// kernel and the left-looking L / U panels eliminate it.  For in <= kLlSub
// this is exactly the reference's inner Crout loop
// (src/lu_nopiv_inner_ll.hxx:197-370); wider blocks nest one more level.
// With lcopy given, the L panels also write their rows' fp16 copies
// (rounded as the fp16 matrix stores them) into the operand copy.
static lu_status ll_block(cudaStream_t st, float* x, int64_t ldx, int64_t n, int64_t ofs,
                          int64_t in, int* first_bad, DevStreams* S, void* lcopy = nullptr,
                          int64_t ldk = 0) {
  for (int64_t c = ofs; c < ofs + in; c += kLlSub) {
    const int64_t w = std::min(kLlSub, ofs + in - c);
    const int64_t rest = n - c - w;
    float* dg = x + c + c * ldx;
    if (c > ofs) {
      // the sub-block's column (st) and row (side stream, when given) are
      // disjoint: their two narrow grids run at once
      const int64_t k = c - ofs;
      const bool side = S != nullptr && rest > 0;
      if (side) LUB_TRY(fork_side(st, S));
      {
        ProfScope ps("sgemm_update", st, 0.0, 2.0 * k * (double)(n - c) * w);
        LUB_TRY(launch_sgemm_update(st, n - c, w, k, -1.0f, x + c + ofs * ldx, ldx,
                                    x + ofs + c * ldx, ldx, 1.0f, dg, ldx, false));
      }
      if (rest > 0) {
        cudaStream_t sr = side ? S->side : st;
        ProfScope ps("sgemm_update", sr, 0.0, 2.0 * k * (double)w * rest);
        LUB_TRY(launch_sgemm_update(sr, w, rest, k, -1.0f, x + c + ofs * ldx, ldx,
                                    x + ofs + (c + w) * ldx, ldx, 1.0f, dg + w * ldx, ldx,
                                    false));
      }
      if (side) LUB_TRY(join_side(st, S));
    }
    {
      ProfScope ps("diag_factor", st, 8.0 * w * w, 2.0 * w * w * (double)w / 3.0);
      LUB_TRY(launch_diag_crout(st, dg, ldx, (int)w, c, first_bad));
    }
    if (rest > 0) {
      ProfScope ps("lupanel", st, 16.0 * rest * w, 2.0 * rest * (double)w * w);
      // lcopy: the finished L rows also go to the fp16 A operand copy
      // (row i, column k at lcopy[i * ldk + k])
      LuPack pk;
      pk.pa = lcopy;
      pk.ldk = ldk;
      pk.row0 = c + w;
      pk.k0 = (int)c;
      LUB_TRY(launch_lupanel(st, dg, ldx, (int)w, rest, rest, true, 0, 0,
                             lcopy ? &pk : nullptr));
    }
  }
  return LU_SUCCESS;
}

// Left-looking (Crout) factorization, restating src/lu_nopiv_ll.hxx:208-575:
// per outer block, one K = ofs update of the block column and the block row
// (FP32 SIMT, or tensor cores on the low-precision copies of all earlier
// factors), then ll_block.  The FP32 path applies every update in the
// reference's order (for nb <= kLlSub).
static lu_status ll_factor(const Plan& p, cudaStream_t st, float* a,
                           int64_t lda, char* ws, int* first_bad, int* err) {
  const int64_t n = p.n, nb = p.nb;
  const bool tc = is_tc(p.outer);
  const TcOperand kind = tc_kind(p.outer);
  const int64_t ldk = (n + 15) / 16 * 16;
  const int64_t es = tc_operand_bytes(kind);
  char* Lc = ws + p.off_lcopy;
  char* Uc = ws + p.off_ucopy;
  DevStreams* S = nullptr;
  LUB_TRY(dev_streams(&S));
  // tensor-core path: as ll_factor_f16, the K range [0, ofs - nb) of block
  // ofs's two updates is computed on the low-priority stream while the
  // previous block is factored (from the L and U copies of the blocks
  // before it), the previous block's own K = nb product after it, and one
  // finishing pass adds the slabs in K order into the fp32 matrix
  auto slabs = [&](int q, int r) {
    return reinterpret_cast<float*>(ws + p.off_part + (size_t)(2 * q + r) * p.part_bytes);
  };
  int early[2][2] = {{0, 0}, {0, 0}};
  auto launch_early = [&](int64_t o) -> lu_status {
    const int q = (int)((o / nb) & 1);
    early[q][0] = early[q][1] = 0;
    const int64_t ke = o - nb;
    if (!tc || o >= n || ke <= 0) return LU_SUCCESS;
    const int64_t in_ = std::min(n - o, nb), updm_ = n - o, rest_ = updm_ - in_;
    const int ks = ll_split(updm_, in_, ke, es);
    ProfScope ps("tc_update", S->update,
                 8.0 * ks * ((double)updm_ * in_ + (double)in_ * rest_) +
                     (double)es * ke * (updm_ + in_ + (rest_ > 0 ? in_ + rest_ : 0)),
                 2.0 * ke * ((double)updm_ * in_ + (double)in_ * rest_));
    LUB_CUDA_TRY(cudaEventRecord(S->ll_ready, st));
    LUB_CUDA_TRY(cudaStreamWaitEvent(S->update, S->ll_ready, 0));
    LUB_TRY(launch_tc_partials(S->update, kind, updm_, in_, ke, Lc + o * ldk * es, ldk,
                               Uc + o * ldk * es, ldk, ks, slabs(q, 0), 0, &early[q][0], err));
    if (rest_ > 0)
      LUB_TRY(launch_tc_partials(S->update, kind, in_, rest_, ke, Lc + o * ldk * es, ldk,
                                 Uc + (o + in_) * ldk * es, ldk, ks, slabs(q, 1), 0,
                                 &early[q][1], err));
    LUB_CUDA_TRY(cudaEventRecord(S->ll_early[q], S->update));
    return LU_SUCCESS;
  };
  for (int64_t ofs = 0; ofs < n; ofs += nb) {
    const int64_t in = std::min(n - ofs, nb);
    const int64_t updm = n - ofs;
    float* blk = a + ofs + ofs * lda;
    const int q = (int)((ofs / nb) & 1);
    LUB_TRY(launch_early(ofs + nb));
    if (ofs > 0) {
      if (tc) {
        // the previous block's own product, then the finishing pass: block
        // column on st, block row on the side stream (disjoint, at once)
        const bool row = updm > in;
        const int64_t k0 = ofs - nb;
        const bool wait_early = early[q][0] > 0 || early[q][1] > 0;
        if (row) LUB_TRY(fork_side(st, S));
        {
          ProfScope ps("tc_update", st,
                       4.0 * (3 + early[q][0]) * updm * in + es * (double)nb * (updm + in),
                       2.0 * nb * (double)updm * in);
          int sl = 0;
          LUB_TRY(launch_tc_partials(st, kind, updm, in, nb, Lc + (ofs * ldk + k0) * es, ldk,
                                     Uc + (ofs * ldk + k0) * es, ldk, 1, slabs(q, 0),
                                     early[q][0], &sl, err));
          if (wait_early) LUB_CUDA_TRY(cudaStreamWaitEvent(st, S->ll_early[q], 0));
          LUB_TRY(launch_splitk_finish(st, updm, in, early[q][0] + sl, slabs(q, 0), -1.0f, blk,
                                       false, lda, nullptr, 0));
        }
        if (row) {
          ProfScope ps("tc_update", S->side,
                       4.0 * (3 + early[q][1]) * in * (updm - in) + es * (double)nb * updm,
                       2.0 * nb * (double)in * (updm - in));
          int sl = 0;
          LUB_TRY(launch_tc_partials(S->side, kind, in, updm - in, nb,
                                     Lc + (ofs * ldk + k0) * es, ldk,
                                     Uc + ((ofs + in) * ldk + k0) * es, ldk, 1, slabs(q, 1),
                                     early[q][1], &sl, err));
          if (wait_early) LUB_CUDA_TRY(cudaStreamWaitEvent(S->side, S->ll_early[q], 0));
          LUB_TRY(launch_splitk_finish(S->side, in, updm - in, early[q][1] + sl, slabs(q, 1),
                                       -1.0f, blk + in * lda, false, lda, nullptr, 0));
          LUB_TRY(join_side(st, S));
        }
      } else {
        // block column and block row at once, as above
        const bool row = updm > in;
        if (row) LUB_TRY(fork_side(st, S));
        {
          ProfScope ps("sgemm_update", st, 0.0, 2.0 * ofs * (double)updm * in);
          LUB_TRY(launch_sgemm_update(st, updm, in, ofs, -1.0f, a + ofs, lda,
                                      a + ofs * lda, lda, 1.0f, blk, lda, false));
        }
        if (row) {
          ProfScope ps("sgemm_update", S->side, 0.0, 2.0 * ofs * (double)in * (updm - in));
          LUB_TRY(launch_sgemm_update(S->side, in, updm - in, ofs, -1.0f, a + ofs, lda,
                                      a + (ofs + in) * lda, lda, 1.0f, blk + in * lda,
                                      lda, false));
          LUB_TRY(join_side(st, S));
        }
      }
    }
    LUB_TRY(ll_block(st, a, lda, n, ofs, in, first_bad, S));
    const int64_t rest = updm - in;
    if (rest > 0 && tc) {
      ProfScope ps("pack_operands", st, 2.0 * rest * in * (4.0 + es));
      // L21 rows [ofs+in, n) of the block's columns -> row-major copy;
      // U12 columns [ofs+in, n) of the block's rows -> column-major copy
      LUB_TRY(launch_pack_a(st, kind, rest, in, blk + in, lda,
                            Lc + ((ofs + in) * ldk + ofs) * es, ldk, nullptr));
      LUB_TRY(launch_pack_b(st, kind, in, rest, blk + in * lda, lda,
                            Uc + ((ofs + in) * ldk + ofs) * es, ldk, nullptr));
    }
  }
  LUB_CUDA_TRY(cudaEventRecord(S->ll_ready, S->update));
  LUB_CUDA_TRY(cudaStreamWaitEvent(st, S->ll_ready, 0));
  return LU_SUCCESS;
}

// Left-looking factorization of an fp16 matrix (the reference's W = fp16
// wrappers, src/lu_nopiv_ll.hxx:646-790).  Per outer block: one K = ofs
// tensor-core update of the block column and the block row read straight
// from the fp16 matrix (U, column-major = K-major) and from a row-major fp16
// copy of the factored L columns, the sum formed in fp32; then the block
// column and row are factored in an fp32 shadow (ll_block) and rounded back
// to fp16.  panel_fp32 = false (OP = fp16): the updated block is stored to
// fp16 once, then copied to the shadow.  panel_fp32 = true (OP = OF = fp32,
// src/lu_nopiv_ll.hxx:172-201): the block is copied to the shadow first
// and the update lands there in fp32, unrounded.  The reference's fp16
// wrappers factor the panel in fp16 arithmetic or with fp16 tensor-core
// inner updates; here the inner elimination always runs in fp32, so its
// results are at least as accurate.
static lu_status ll_factor_f16(const Plan& p, cudaStream_t st, __half* a, int64_t lda,
                               char* ws, int* first_bad, int* err) {
  const int64_t n = p.n, nb = p.nb;
  const int64_t ldk = (n + 15) / 16 * 16;
  char* Lc = ws + p.off_lcopy;
  float* Sh = reinterpret_cast<float*>(ws + p.off_shadow);
  const int64_t lds = p.ld_shadow;
  DevStreams* S = nullptr;
  LUB_TRY(dev_streams(&S));
  // partial-product slabs of the block column (r = 0) and block row (r = 1)
  // updates of the blocks of parity q
  auto slabs = [&](int q, int r) {
    return reinterpret_cast<float*>(ws + p.off_part + (size_t)(2 * q + r) * p.part_bytes);
  };
  int early[2][2] = {{0, 0}, {0, 0}};  // slabs computed ahead, per parity / update
  // Block column o's updates over K = [0, o - nb) (all factored columns but
  // the previous block's), on the low-priority stream while the previous
  // block is factored on st.  Everything they read is final once the block
  // before the previous one is done: the L copy's columns [0, o - nb) and
  // the U rows [0, o - nb) of the fp16 matrix.
  auto launch_early = [&](int64_t o) -> lu_status {
    const int q = (int)((o / nb) & 1);
    early[q][0] = early[q][1] = 0;
    const int64_t ke = o - nb;
    if (o >= n || ke <= 0) return LU_SUCCESS;
    const int64_t in_ = std::min(n - o, nb), updm_ = n - o, rest_ = updm_ - in_;
    const int ks = ll_split(updm_, in_, ke, 2);
    ProfScope ps("tc_update", S->update,
                 8.0 * (ks * (double)updm_ * in_ + (rest_ > 0 ? ks * (double)in_ * rest_ : 0.0)) +
                     2.0 * (double)ke * (updm_ + in_ + (rest_ > 0 ? in_ + rest_ : 0)),
                 2.0 * ke * ((double)updm_ * in_ + (double)in_ * rest_));
    LUB_CUDA_TRY(cudaEventRecord(S->ll_ready, st));
    LUB_CUDA_TRY(cudaStreamWaitEvent(S->update, S->ll_ready, 0));
    LUB_TRY(launch_tc_partials(S->update, TcOperand::F16, updm_, in_, ke, Lc + o * ldk * 2, ldk,
                               a + o * lda, lda, ks, slabs(q, 0), 0, &early[q][0], err));
    if (rest_ > 0)
      LUB_TRY(launch_tc_partials(S->update, TcOperand::F16, in_, rest_, ke, Lc + o * ldk * 2, ldk,
                                 a + (o + in_) * lda, lda, ks, slabs(q, 1), 0, &early[q][1],
                                 err));
    LUB_CUDA_TRY(cudaEventRecord(S->ll_early[q], S->update));
    return LU_SUCCESS;
  };
  for (int64_t ofs = 0; ofs < n; ofs += nb) {
    const int64_t in = std::min(n - ofs, nb);
    const int64_t updm = n - ofs;
    const int64_t rest = updm - in;
    const int q = (int)((ofs / nb) & 1);
    __half* blk = a + ofs + ofs * lda;
    float* sblk = Sh + ofs + ofs * lds;
    // the next block's early products, beside this block's work
    LUB_TRY(launch_early(ofs + nb));
    auto to_shadow = [&]() -> lu_status {
      ProfScope ps("convert", st, 6.0 * (double)in * (updm + rest));
      LUB_TRY(launch_convert(st, updm, in, blk, LU_F16, lda, sblk, LU_F32, lds, 0));
      if (rest > 0)
        LUB_TRY(launch_convert(st, in, rest, blk + in * lda, LU_F16, lda, sblk + in * lds,
                               LU_F32, lds, 0));
      return LU_SUCCESS;
    };
    if (p.panel_fp32 || ofs == 0) LUB_TRY(to_shadow());
    if (ofs > 0) {
      // the previous block's own product (K range [ofs - nb, ofs)), then the
      // sum of all slabs in K order: block column on st, block row on the
      // side stream (disjoint, at once).  panel_fp32: the update lands in
      // the shadow; otherwise in the fp16 matrix (one rounding), and the
      // finishing kernel also writes the stored values to the shadow
      const int64_t k0 = ofs - nb;
      const bool wait_early = early[q][0] > 0 || early[q][1] > 0;
      if (rest > 0) LUB_TRY(fork_side(st, S));
      {
        ProfScope ps("tc_update", st, 4.0 * (2 + early[q][0]) * updm * in + 2.0 * (double)nb * (updm + in),
                     2.0 * nb * (double)updm * in);
        int sl = 0;
        LUB_TRY(launch_tc_partials(st, TcOperand::F16, updm, in, nb, Lc + (ofs * ldk + k0) * 2,
                                   ldk, a + k0 + ofs * lda, lda, 1, slabs(q, 0), early[q][0], &sl,
                                   err));
        if (wait_early) LUB_CUDA_TRY(cudaStreamWaitEvent(st, S->ll_early[q], 0));
        LUB_TRY(launch_splitk_finish(st, updm, in, early[q][0] + sl, slabs(q, 0), -1.0f,
                                     p.panel_fp32 ? (void*)sblk : (void*)blk, !p.panel_fp32,
                                     p.panel_fp32 ? lds : lda,
                                     p.panel_fp32 ? nullptr : sblk, lds));
      }
      if (rest > 0) {
        ProfScope ps("tc_update", S->side,
                     4.0 * (2 + early[q][1]) * in * rest + 2.0 * (double)nb * (in + rest),
                     2.0 * nb * (double)in * rest);
        int sl = 0;
        LUB_TRY(launch_tc_partials(S->side, TcOperand::F16, in, rest, nb,
                                   Lc + (ofs * ldk + k0) * 2, ldk, a + k0 + (ofs + in) * lda, lda,
                                   1, slabs(q, 1), early[q][1], &sl, err));
        if (wait_early) LUB_CUDA_TRY(cudaStreamWaitEvent(S->side, S->ll_early[q], 0));
        LUB_TRY(launch_splitk_finish(S->side, in, rest, early[q][1] + sl, slabs(q, 1), -1.0f,
                                     p.panel_fp32 ? (void*)(sblk + in * lds)
                                                  : (void*)(blk + in * lda),
                                     !p.panel_fp32, p.panel_fp32 ? lds : lda,
                                     p.panel_fp32 ? nullptr : sblk + in * lds, lds));
        LUB_TRY(join_side(st, S));
      }
    }
    // (the L panels write the L operand copy of the rows below the block)
    LUB_TRY(ll_block(st, Sh, lds, n, ofs, in, first_bad, S, Lc, ldk));
    {
      ProfScope ps("convert", st, 6.0 * (double)in * (updm + rest));
      LUB_TRY(launch_convert(st, updm, in, sblk, LU_F32, lds, blk, LU_F16, lda, 0));
      if (rest > 0)
        LUB_TRY(launch_convert(st, in, rest, sblk + in * lds, LU_F32, lds, blk + in * lda,
                               LU_F16, lda, 0));
    }
  }
  // the low-priority stream joins the caller's stream
  LUB_CUDA_TRY(cudaEventRecord(S->ll_ready, S->update));
  LUB_CUDA_TRY(cudaStreamWaitEvent(st, S->ll_ready, 0));
  return LU_SUCCESS;
}

// The internal streams and events of a device (dev_streams) are shared by
// every call on it, so one host thread at a time enqueues a factorization
// on a device: each call's work is queued whole, with its events recorded
// and waited for under this lock, and calls from several threads run one
// after another on the internal streams.
static std::mutex& device_mutex() {
  static std::mutex mu[64];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) dev = 0;
  return mu[dev & 63];
}

lu_status factorize(const lu_opts& o, cudaStream_t st, int64_t m, int64_t n,
                    void* d_a, lu_dtype dtype_a, int64_t lda, int* d_info,
                    void* d_a_lowp, int64_t ld_lowp, void* workspace,
                    size_t ws_bytes) {
  if (m < 0 || n < 0) return LU_ERR_INVALID_ARG;
  if (lda < std::max<int64_t>(1, m)) return LU_ERR_INVALID_ARG;
  if (d_info == nullptr) return LU_ERR_INVALID_ARG;
  if (n > 0 && d_a == nullptr) return LU_ERR_INVALID_ARG;
  if (d_a_lowp != nullptr && ld_lowp < std::max<int64_t>(1, m))
    return LU_ERR_INVALID_ARG;
  Plan p;
  LUB_TRY(make_plan(o, m, n, dtype_a, &p));
  // fp16 storage: the tensor cores read U straight from the matrix
  if (dtype_a == LU_F16 && n > 0 &&
      ((uintptr_t)d_a % 16 != 0 || lda % 8 != 0 || d_a_lowp != nullptr))
    return LU_ERR_INVALID_ARG;
  LUB_TRY(check_device());
  if (workspace != nullptr && ws_bytes < p.ws_bytes) return LU_ERR_WORKSPACE;
  std::lock_guard<std::mutex> lock(device_mutex());

  void* ws = workspace;
  bool owned = false;
  if (ws == nullptr) {
    if (pool_malloc_async((void**)&ws, p.ws_bytes, st) != cudaSuccess) return LU_ERR_ALLOC;
    owned = true;
  }
  char* wsb = static_cast<char*>(ws);
  int* first_bad = reinterpret_cast<int*>(wsb + p.off_status);
  int* err = first_bad + 1;
  lu_status s = launch_fill_int(st, first_bad, kNoBadPivot, 1);
  if (s == LU_SUCCESS) s = launch_fill_int(st, err, 0, 1);
  if (s == LU_SUCCESS && n > 0)
    s = dtype_a == LU_F16
            ? ll_factor_f16(p, st, static_cast<__half*>(d_a), lda, wsb, first_bad, err)
        : p.variant == LU_LEFT_LOOKING
            ? ll_factor(p, st, static_cast<float*>(d_a), lda, wsb, first_bad, err)
            : rl_factor(p, st, static_cast<float*>(d_a), lda, wsb, first_bad, err);
  if (s == LU_SUCCESS) s = launch_finalize_info(st, first_bad, err, d_info);
  if (s == LU_SUCCESS && d_a_lowp != nullptr && n > 0)
    s = launch_convert(st, m, n, d_a, LU_F32, lda, d_a_lowp, LU_F16, ld_lowp, 0);
  if (owned) cudaFreeAsync(ws, st);
  return s;
}

// Host-memory entry.  The matrix goes in by column chunks of whole outer
// blocks on one copy stream while the device works: each chunk, once in,
// receives the steps of the earlier chunks (catch_up, beside the
// factorization of the previous chunk), then its own steps run (rl_factor
// restricted to it), each sending its finished block column back on a
// second copy stream while the factorization goes on.
// Every element receives the same operations in the same order as in the
// device-memory entry, so the factors are bit-identical to it.
lu_status factorize_host(const lu_opts& o, cudaStream_t st, int64_t n, float* h_a,
                         int64_t lda, float* d_a, int64_t ldda, int* d_info,
                         void* workspace, size_t ws_bytes) {
  if (n < 0 || lda < std::max<int64_t>(1, n) || ldda < std::max<int64_t>(1, n))
    return LU_ERR_INVALID_ARG;
  if (d_info == nullptr) return LU_ERR_INVALID_ARG;
  if (n > 0 && (h_a == nullptr || d_a == nullptr)) return LU_ERR_INVALID_ARG;
  if (o.variant != LU_RIGHT_LOOKING) return LU_ERR_UNSUPPORTED;
  Plan p;
  LUB_TRY(make_plan(o, n, n, LU_F32, &p));
  LUB_TRY(check_device());
  if (workspace != nullptr && ws_bytes < p.ws_bytes) return LU_ERR_WORKSPACE;
  std::lock_guard<std::mutex> lock(device_mutex());
  void* ws = workspace;
  bool owned = false;
  if (ws == nullptr) {
    if (pool_malloc_async((void**)&ws, p.ws_bytes, st) != cudaSuccess) return LU_ERR_ALLOC;
    owned = true;
  }
  char* wsb = static_cast<char*>(ws);
  int* first_bad = reinterpret_cast<int*>(wsb + p.off_status);
  int* err = first_bad + 1;
  lu_status s = launch_fill_int(st, first_bad, kNoBadPivot, 1);
  if (s == LU_SUCCESS) s = launch_fill_int(st, err, 0, 1);
  const int64_t nb = p.nb;
  const bool tc = is_tc(p.outer);
  const TcOperand kind = tc_kind(p.outer);
  const int64_t nblk = ceil_div(std::max<int64_t>(n, 1), nb);
  // Column chunks of whole outer blocks: four with the step-order catch-up
  // (B200 at n = 16384: 4 chunks 40 ms, 2 or 3 chunks 41-42 ms, 8 chunks 46
  // ms, one 47 ms); kLlChunks with the left-looking one, whose chain per
  // earlier step is short, so a smaller last chunk -- less left to do and
  // to send back after the last rows arrive -- wins.
  const bool ll_order = p.lookahead && tc && !tc_scaled(kind) && p.bulk_group >= 2;
  const int64_t cw = ceil_div(nblk, ll_order ? kLlChunks : 4) * nb;
  const bool chunked = n > 2 * nb && !(tc && tc_scaled(kind) && nb % 128 != 0) &&
                       ceil_div(n, cw) <= kMaxChunks;
  auto h2d = [&](cudaStream_t sm, int64_t c0, int64_t c1) {
    return cudaMemcpy2DAsync(d_a + c0 * ldda, (size_t)ldda * 4, h_a + c0 * lda,
                             (size_t)lda * 4, (size_t)n * 4, (size_t)(c1 - c0),
                             cudaMemcpyHostToDevice, sm);
  };
  auto d2h = [&](cudaStream_t sm, int64_t c0, int64_t c1) {
    return cudaMemcpy2DAsync(h_a + c0 * lda, (size_t)lda * 4, d_a + c0 * ldda,
                             (size_t)ldda * 4, (size_t)n * 4, (size_t)(c1 - c0),
                             cudaMemcpyDeviceToHost, sm);
  };
  if (s == LU_SUCCESS && n > 0 && !chunked) {
    if (h2d(st, 0, n) != cudaSuccess) s = LU_ERR_CUDA;
    if (s == LU_SUCCESS) s = rl_factor(p, st, d_a, ldda, wsb, first_bad, err);
    if (s == LU_SUCCESS && d2h(st, 0, n) != cudaSuccess) s = LU_ERR_CUDA;
  } else if (s == LU_SUCCESS && n > 0) {
    DevStreams* S = nullptr;
    s = dev_streams(&S);
    TcWs wk;
    if (tc) wk = tc_ws_layout(256, n - nb, n - nb, nb, kind);
    cudaStream_t ci = S ? S->copy : nullptr, co = S ? S->copy_out : nullptr;
    ColumnSink sink;
    sink.h = h_a;
    sink.ldh = lda;
    sink.out = co;
    auto ok = [&](cudaError_t e) {
      if (e != cudaSuccess && s == LU_SUCCESS) s = LU_ERR_CUDA;
      return s == LU_SUCCESS;
    };
    // Under look-ahead rl_factor marks each step's finished block column
    // with an event, and the catch-up of an arrived chunk runs on its own
    // stream beside the factorization of the chunk before it (with its own
    // operand buffers, two: see catch_up); otherwise the catch-up runs in
    // order on the stream.
    const bool la = p.lookahead && n > 2 * nb && !(tc && tc_scaled(kind) && nb % 128 != 0);
    cudaStream_t cu = la && S ? S->catchup : st;
    TcWs wcu[2] = {wk, wk};
    char* cubuf = wsb;
    void* cu_alloc = nullptr;
    // several steps per bulk pass: the left-looking catch-up (catch_up_ll);
    // one pass per step keeps the step-by-step order of the device entry
    const bool llc = la && tc && !tc_scaled(kind) && p.bulk_group >= 2;
    if (llc && S) cu = S->catchup_chain;  // the chain of block rows comes first
    LlCatchup llb;
    if (s == LU_SUCCESS && llc) {
      const int64_t c_last = (ceil_div(n, cw) - 1) * cw;  // first column of the last chunk
      const int64_t es = tc_operand_bytes(kind);
      llb.ldl = align_up(c_last, 64);
      llb.ldx = llb.ldl;
      llb.ksplit_max = kLlCatchupSplitMax;
      const size_t lp_bytes = align_up((size_t)n * llb.ldl * es, 1024);
      const size_t xp_bytes = align_up((size_t)llb.ldx * cw * es, 1024);
      llb.slab = splitk_slab_floats(nb, cw);
      // two sets of slabs: a block row's partial products stay until its
      // solve has read them while the next row's are computed
      const size_t part_bytes = 2 * (size_t)kLlCatchupSplitMax * llb.slab * 4;
      if (pool_malloc_async((void**)&cu_alloc, lp_bytes + xp_bytes + part_bytes, st) !=
          cudaSuccess)
        s = LU_ERR_ALLOC;
      llb.lp = static_cast<char*>(cu_alloc);
      llb.xp = llb.lp + lp_bytes;
      llb.part = reinterpret_cast<float*>(llb.xp + xp_bytes);
      // the factorization's panels write the L columns left of the last
      // chunk into lp as they finish them (no packing pass)
      sink.lp = llb.lp;
      sink.ldl = llb.ldl;
      sink.lp_cols = c_last;
    } else if (s == LU_SUCCESS && la && tc) {
      wcu[0] = tc_ws_layout(0, n - nb, n - nb, nb, kind);
      wcu[1] = tc_ws_layout(wcu[0].bytes, n - nb, n - nb, nb, kind);
      if (pool_malloc_async((void**)&cu_alloc, wcu[0].bytes + wcu[1].bytes, st) != cudaSuccess)
        s = LU_ERR_ALLOC;
      cubuf = static_cast<char*>(cu_alloc);
    }
    if (s == LU_SUCCESS && ok(cudaEventRecord(S->fork, st)) &&
        ok(cudaStreamWaitEvent(ci, S->fork, 0)) && ok(cudaStreamWaitEvent(co, S->fork, 0)) &&
        (!la || ok(cudaStreamWaitEvent(cu, S->fork, 0)))) {
      int q = 0;
      for (int64_t c0 = 0; c0 < n && s == LU_SUCCESS; c0 += cw, ++q) {
        const int64_t c1 = std::min(n, c0 + cw);
        if (llc && q > 0) {
          // the rows above c0 first: the chunk's catch-up chain starts on
          // them while its lower rows are still on the way
          {
            ProfScope ps("copy_h2d", ci, 4.0 * (double)c0 * (c1 - c0));
            if (!ok(cudaMemcpy2DAsync(d_a + c0 * ldda, (size_t)ldda * 4, h_a + c0 * lda,
                                      (size_t)lda * 4, (size_t)c0 * 4, (size_t)(c1 - c0),
                                      cudaMemcpyHostToDevice, ci)))
              break;
          }
          if (!ok(cudaEventRecord(S->chunk_top[q], ci))) break;
          ProfScope ps("copy_h2d", ci, 4.0 * (double)(n - c0) * (c1 - c0));
          if (!ok(cudaMemcpy2DAsync(d_a + c0 + c0 * ldda, (size_t)ldda * 4, h_a + c0 + c0 * lda,
                                    (size_t)lda * 4, (size_t)(n - c0) * 4, (size_t)(c1 - c0),
                                    cudaMemcpyHostToDevice, ci)))
            break;
        } else {
          ProfScope ps("copy_h2d", ci, 4.0 * (double)n * (c1 - c0));
          if (!ok(h2d(ci, c0, c1))) break;
        }
        if (!ok(cudaEventRecord(S->chunk_in[q], ci))) break;
      }
      q = 0;
      for (int64_t c0 = 0; c0 < n && s == LU_SUCCESS; c0 += cw, ++q) {
        const int64_t c1 = std::min(n, c0 + cw);
        if (!ok(cudaStreamWaitEvent(cu, llc && q > 0 ? S->chunk_top[q] : S->chunk_in[q], 0)))
          break;
        if (q > 0 && llc) {
          // (its rows above c0 go out group by group inside)
          if ((s = catch_up_ll(p, cu, d_a, ldda, &llb, err, c0, c1, S, sink, S->chunk_in[q])) !=
              LU_SUCCESS)
            break;
        } else if (q > 0) {
          s = catch_up(p, cu, d_a, ldda, cubuf, wcu, err, c0, c1, la ? S : nullptr);
          if (s != LU_SUCCESS) break;
          // the rows [0, c0) of the chunk are final now: out at once, ahead
          // of the chunk's own steps (which send the rows [c0, n) of each
          // block column as it finishes)
          if (!ok(cudaEventRecord(S->cu_out, cu)) || !ok(cudaStreamWaitEvent(co, S->cu_out, 0)))
            break;
          ProfScope ps("copy_d2h", co, 4.0 * (double)c0 * (c1 - c0));
          if (!ok(cudaMemcpy2DAsync(h_a + c0 * lda, (size_t)lda * 4, d_a + c0 * ldda,
                                    (size_t)ldda * 4, (size_t)c0 * 4, (size_t)(c1 - c0),
                                    cudaMemcpyDeviceToHost, co)))
            break;
        }
        if (la && (!ok(cudaEventRecord(S->cu_done, cu)) ||
                   !ok(cudaStreamWaitEvent(st, S->cu_done, 0))))
          break;
        if ((s = rl_factor(p, st, d_a, ldda, wsb, first_bad, err, c0, c1, &sink)) != LU_SUCCESS)
          break;
      }
      // join the side streams (also on the error path)
      if (la) {
        cudaEventRecord(S->cu_done, cu);
        cudaStreamWaitEvent(st, S->cu_done, 0);
        cudaEventRecord(S->cu_join, S->catchup_bulk);
        cudaStreamWaitEvent(st, S->cu_join, 0);
        if (llc) {
          cudaEventRecord(S->cu_join, S->catchup_early);
          cudaStreamWaitEvent(st, S->cu_join, 0);
        }
      }
      cudaEventRecord(S->out_done, co);
      cudaStreamWaitEvent(st, S->out_done, 0);
      cudaEventRecord(S->copied, ci);
      cudaStreamWaitEvent(st, S->copied, 0);
    }
    if (cu_alloc) cudaFreeAsync(cu_alloc, st);
  }
  if (s == LU_SUCCESS) s = launch_finalize_info(st, first_bad, err, d_info);
  if (owned) cudaFreeAsync(ws, st);
  return s;
}

lu_status gemm_update(lu_compute compute, cudaStream_t st, int64_t m, int64_t n,
                      int64_t k, double alpha, const float* a, int64_t lda,
                      const float* b, int64_t ldb, double beta, float* c,
                      int64_t ldc, void* workspace, size_t ws_bytes) {
  if (compute == LU_COMPUTE_FP32)
    return launch_sgemm_update(st, m, n, k, (float)alpha, a, lda, b, ldb,
                               (float)beta, c, ldc, false);
  if (!is_tc(compute)) return LU_ERR_UNSUPPORTED;
  if (beta != 1.0) return LU_ERR_UNSUPPORTED;  // the update form C += alpha*A*B
  if (k <= 0) return LU_SUCCESS;
  const TcWs w = tc_ws_layout(256, m, n, k, tc_kind(compute));
  const size_t need = 256 + w.bytes;
  if (workspace != nullptr && ws_bytes < need) return LU_ERR_WORKSPACE;
  void* ws = workspace;
  bool owned = false;
  if (ws == nullptr) {
    if (pool_malloc_async((void**)&ws, need, st) != cudaSuccess) return LU_ERR_ALLOC;
    owned = true;
  }
  char* wsb = static_cast<char*>(ws);
  int* err = reinterpret_cast<int*>(wsb);
  lu_status s = launch_fill_int(st, err, 0, 1);
  if (s == LU_SUCCESS)
    s = tc_update_fp32(st, tc_kind(compute), m, n, k, (float)alpha, a, lda, b,
                       ldb, c, ldc, wsb, w, err);
  if (owned) cudaFreeAsync(ws, st);
  return s;
}

// gemmex with operand / result storage types (the reference's gemmex
// instantiations, src/gemm.cu:17-316): fp32 operands and result on the SIMT
// fp32 path or any tensor-core kind as gemm_update; fp16 operands and / or an
// fp16 result on the tensor cores with fp16 operands and fp32 accumulation
// (LU_COMPUTE_TC32, and TC16 / FP16, whose fp16 accumulation the tensor
// cores replace by fp32 accumulation with one rounding of the result).
lu_status gemm_update_ex(lu_compute compute, cudaStream_t st, int64_t m, int64_t n,
                         int64_t k, double alpha, const void* a, lu_dtype ta, int64_t lda,
                         const void* b, lu_dtype tb, int64_t ldb, double beta, void* c,
                         lu_dtype tc, int64_t ldc, void* workspace, size_t ws_bytes) {
  const bool f32ops = ta == LU_F32 && tb == LU_F32;
  const bool f16ops = ta == LU_F16 && tb == LU_F16;
  if ((!f32ops && !f16ops) || (tc != LU_F32 && tc != LU_F16)) return LU_ERR_UNSUPPORTED;
  if (compute == LU_COMPUTE_FP32) {
    if (!f32ops || tc != LU_F32) return LU_ERR_UNSUPPORTED;
    return gemm_update(compute, st, m, n, k, alpha, (const float*)a, lda, (const float*)b,
                       ldb, beta, (float*)c, ldc, workspace, ws_bytes);
  }
  const lu_compute kc = (compute == LU_COMPUTE_FP16 || compute == LU_COMPUTE_TC16)
                            ? LU_COMPUTE_TC32 : compute;
  if (!is_tc(kc)) return LU_ERR_UNSUPPORTED;
  if (f32ops && tc == LU_F32)
    return gemm_update(kc, st, m, n, k, alpha, (const float*)a, lda, (const float*)b, ldb,
                       beta, (float*)c, ldc, workspace, ws_bytes);
  if (kc != LU_COMPUTE_TC32) return LU_ERR_UNSUPPORTED;  // fp16 data: fp16 operands
  if (beta != 1.0) return LU_ERR_UNSUPPORTED;  // the update form C += alpha*A*B
  if (k <= 0) return LU_SUCCESS;
  const TcWs w = tc_ws_layout(256, m, n, k, TcOperand::F16);
  const size_t need = 256 + w.bytes;
  if (workspace != nullptr && ws_bytes < need) return LU_ERR_WORKSPACE;
  void* ws = workspace;
  bool owned = false;
  if (ws == nullptr) {
    if (pool_malloc_async((void**)&ws, need, st) != cudaSuccess) return LU_ERR_ALLOC;
    owned = true;
  }
  char* wsb = static_cast<char*>(ws);
  int* err = reinterpret_cast<int*>(wsb);
  const int64_t ldk = tc_packed_k(TcOperand::F16, k);
  __half* ap = reinterpret_cast<__half*>(wsb + w.off_a);
  __half* bp = reinterpret_cast<__half*>(wsb + w.off_b);
  lu_status s = launch_fill_int(st, err, 0, 1);
  if (s == LU_SUCCESS) {
    ProfScope ps("pack_operands", st, (double)(m + n) * (double)k * (f16ops ? 4.0 : 6.0));
    if (f16ops) {
      s = launch_pack_a_f16(st, m, k, (const __half*)a, lda, ap, ldk);
      if (s == LU_SUCCESS) s = launch_pack_b_f16(st, k, n, (const __half*)b, ldb, bp, ldk);
    } else {
      s = tc_pack(st, TcOperand::F16, m, n, k, (const float*)a, lda, (const float*)b, ldb,
                  wsb, w);
    }
  }
  if (s == LU_SUCCESS) {
    ProfScope ps("tc_update", st, (tc == LU_F32 ? 8.0 : 4.0) * m * n + 2.0 * (m + n) * k,
                 2.0 * m * n * k);
    s = tc == LU_F32 ? launch_tc_update(st, TcOperand::F16, m, n, k, (float)alpha, ap, ldk,
                                        bp, ldk, (float*)c, ldc, nullptr, nullptr, err)
                     : launch_tc_update_h(st, TcOperand::F16, m, n, k, (float)alpha, ap, ldk,
                                          bp, ldk, (__half*)c, ldc, err);
  }
  if (owned) cudaFreeAsync(ws, st);
  return s;
}

}  // namespace lub
