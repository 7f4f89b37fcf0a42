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

#include <algorithm>

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
         c == LU_COMPUTE_TC32_E4M3;
}

static TcOperand tc_kind(lu_compute c) {
  return c == LU_COMPUTE_TC32_BF16 ? TcOperand::BF16
       : c == LU_COMPUTE_TC32_E4M3 ? TcOperand::E4M3
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
  const int64_t ldk = (K + 15) / 16 * 16;
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

// C (fp32) -= A * B through the tensor cores: pack A (column-major fp32,
// lda) and B (column-major fp32, ldb) into the workspace, then update.
static lu_status tc_update_fp32(cudaStream_t st, TcOperand kind, int64_t M,
                                int64_t N, int64_t K, float alpha,
                                const float* a, int64_t lda, const float* b,
                                int64_t ldb, float* c, int64_t ldc, char* ws,
                                const TcWs& w, int* err) {
  const int64_t ldk = (K + 15) / 16 * 16;
  void* ap = ws + w.off_a;
  void* bp = ws + w.off_b;
  int* sa = nullptr;
  int* sb = nullptr;
  if (kind == TcOperand::E4M3) {
    sa = reinterpret_cast<int*>(ws + w.off_sa);
    sb = reinterpret_cast<int*>(ws + w.off_sb);
    int* tmp = reinterpret_cast<int*>(ws + w.off_tmp);
    LUB_TRY(launch_scale_rowtiles(st, M, K, a, lda, sa, tmp));
    LUB_TRY(launch_scale_coltiles(st, K, N, b, ldb, sb, tmp));
  }
  const double es = tc_operand_bytes(kind);
  {
    ProfScope ps("pack_operands", st, (double)(M + N) * K * (4.0 + es));
    LUB_TRY(launch_pack_a(st, kind, M, K, a, lda, ap, ldk, sa));
    LUB_TRY(launch_pack_b(st, kind, K, N, b, ldb, bp, ldk, sb));
  }
  // algorithmic bytes: C read + written once (fp32), both operands read once
  ProfScope ps("tc_update", st, 8.0 * M * N + es * (double)(M + N) * K,
               2.0 * M * N * K);
  return launch_tc_update(st, kind, M, N, K, alpha, ap, ldk, bp, ldk, c, ldc,
                          sa, sb, err);
}

lu_status make_plan(const lu_opts& o, int64_t m, int64_t n, lu_dtype dtype,
                    Plan* p) {
  if (m != n) return LU_ERR_UNSUPPORTED;
  if (n < 0) return LU_ERR_INVALID_ARG;
  if (o.ib != 8) return LU_ERR_UNSUPPORTED;
  if (o.nb < 8 || o.nb % 8 != 0 || o.nb > 4096) return LU_ERR_INVALID_ARG;
  const int dw = o.diag_width == 0 ? 128 : o.diag_width;
  if (dw < 8 || dw > 128 || dw % 8 != 0) return LU_ERR_INVALID_ARG;
  if (dtype != LU_F32) return LU_ERR_UNSUPPORTED;
  if (o.variant != LU_RIGHT_LOOKING) return LU_ERR_UNSUPPORTED;
  if (o.inner_update != LU_COMPUTE_FP32) return LU_ERR_UNSUPPORTED;
  if (o.outer_update != LU_COMPUTE_FP32 && !is_tc((lu_compute)o.outer_update))
    return LU_ERR_UNSUPPORTED;
  p->n = n;
  p->nb = o.nb;
  p->diag_w = (int)std::min<int64_t>(dw, o.nb);
  p->inner = (lu_compute)o.inner_update;
  p->outer = (lu_compute)o.outer_update;
  p->variant = (lu_variant)o.variant;
  p->lookahead = o.lookahead != 0;
  p->dtype = dtype;
  size_t off = 0;
  p->off_status = off;  // [0] first bad pivot, [1] device wait error
  off += 256;
  if (is_tc(p->outer) && n > p->nb) {
    const int64_t t = n - p->nb;
    TcWs w = tc_ws_layout(off, t, t, p->nb, tc_kind(p->outer));
    p->off_lcopy = w.off_a;
    off += w.bytes;
  }
  p->ws_bytes = off;
  return LU_SUCCESS;
}

// Factor the outer block column/row starting at (ofs, ofs): width `in`,
// `updm` rows (and columns) remaining.
static lu_status factor_block(const Plan& p, cudaStream_t st, float* a,
                              int64_t lda, int64_t ofs, int64_t in,
                              int64_t updm, int* first_bad) {
  float* blk = a + ofs + ofs * lda;
  for (int64_t p0 = 0; p0 < in; p0 += p.diag_w) {
    const int w = (int)std::min<int64_t>(in - p0, p.diag_w);
    float* dg = blk + p0 + p0 * lda;
    {
      ProfScope ps("diag_factor", st, 8.0 * w * w, 2.0 * w * w * w / 3.0);
      LUB_TRY(launch_diag_factor(st, dg, lda, w, ofs + p0, first_bad));
    }
    const int64_t rest = updm - (p0 + w);
    if (rest > 0) {
      ProfScope ps("lupanel", st, 2.0 * 8.0 * rest * w, 2.0 * rest * (double)w * w);
      LUB_TRY(launch_lupanel(st, dg, lda, w, rest, rest));
    }
    if (p0 + w < in) {
      ProfScope ps("sgemm_chunk8", st, 0.0,
                   2.0 * w * ((double)(updm - p0 - w) * (in - p0 - w) +
                              (double)(in - p0 - w) * (updm - in)));
      // rest of the outer block column: rows [p0+w, updm), cols [p0+w, in)
      LUB_TRY(launch_sgemm_update(st, updm - (p0 + w), in - (p0 + w), w, -1.0f,
                                  dg + w, lda, dg + (int64_t)w * lda, lda, 1.0f,
                                  dg + w + (int64_t)w * lda, lda, true));
      // rest of the outer block row: rows [p0+w, in), cols [in, updm)
      if (updm > in)
        LUB_TRY(launch_sgemm_update(st, in - (p0 + w), updm - in, w, -1.0f,
                                    dg + w, lda, blk + p0 + in * lda, lda, 1.0f,
                                    blk + (p0 + w) + in * lda, lda, true));
    }
  }
  return LU_SUCCESS;
}

static lu_status rl_factor(const Plan& p, cudaStream_t st, float* a,
                           int64_t lda, char* ws, int* first_bad, int* err) {
  const int64_t n = p.n, nb = p.nb;
  TcWs w;
  if (is_tc(p.outer) && n > nb) w = tc_ws_layout(256, n - nb, n - nb, nb, tc_kind(p.outer));
  for (int64_t ofs = 0; ofs < n; ofs += nb) {
    const int64_t in = std::min(n - ofs, nb);
    const int64_t updm = n - ofs;
    LUB_TRY(factor_block(p, st, a, lda, ofs, in, updm, first_bad));
    const int64_t ofst = ofs + nb;
    const int64_t tn = n - ofst;
    if (tn <= 0) continue;
    if (is_tc(p.outer)) {
      // TC32 outer update (src/lu_nopiv.hxx:155-183): rounded copies of
      // L21 and U12, fp32 accumulation, C -= acc in fp32.
      LUB_TRY(tc_update_fp32(st, tc_kind(p.outer), tn, tn, nb, -1.0f,
                             a + ofst + ofs * lda, lda, a + ofs + ofst * lda, lda,
                             a + ofst + ofst * lda, lda, ws, w, err));
    } else {
      ProfScope ps("sgemm_update", st, 8.0 * tn * tn, 2.0 * tn * tn * (double)nb);
      LUB_TRY(launch_sgemm_update(st, tn, tn, nb, -1.0f, a + ofst + ofs * lda,
                                  lda, a + ofs + ofst * lda, lda, 1.0f,
                                  a + ofst + ofst * lda, lda, false));
    }
  }
  return LU_SUCCESS;
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
  LUB_TRY(check_device());
  if (workspace != nullptr && ws_bytes < p.ws_bytes) return LU_ERR_WORKSPACE;

  void* ws = workspace;
  bool owned = false;
  if (ws == nullptr) {
    if (cudaMallocAsync(&ws, p.ws_bytes, st) != cudaSuccess) return LU_ERR_ALLOC;
    owned = true;
  }
  char* wsb = static_cast<char*>(ws);
  int* first_bad = reinterpret_cast<int*>(wsb + p.off_status);
  int* err = first_bad + 1;
  lu_status s = launch_fill_int(st, first_bad, kNoBadPivot, 1);
  if (s == LU_SUCCESS) s = launch_fill_int(st, err, 0, 1);
  if (s == LU_SUCCESS && n > 0)
    s = rl_factor(p, st, static_cast<float*>(d_a), lda, wsb, first_bad, err);
  if (s == LU_SUCCESS) s = launch_finalize_info(st, first_bad, err, d_info);
  if (s == LU_SUCCESS && d_a_lowp != nullptr && n > 0)
    s = launch_convert(st, m, n, d_a, LU_F32, lda, d_a_lowp, LU_F16, ld_lowp, 0);
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
    if (cudaMallocAsync(&ws, need, st) != cudaSuccess) return LU_ERR_ALLOC;
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

}  // namespace lub
