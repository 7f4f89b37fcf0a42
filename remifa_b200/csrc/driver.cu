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
         c == LU_COMPUTE_TC32_E4M3 || c == LU_COMPUTE_TC32_SPLIT ||
         c == LU_COMPUTE_TC16;
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
  if (is_tc((lu_compute)o.outer_update)) return LU_ERR_UNSUPPORTED;  // not yet
  p->n = n;
  p->nb = o.nb;
  p->diag_w = (int)std::min<int64_t>(dw, o.nb);
  p->inner = (lu_compute)o.inner_update;
  p->outer = (lu_compute)o.outer_update;
  p->variant = (lu_variant)o.variant;
  p->lookahead = o.lookahead != 0;
  p->dtype = dtype;
  size_t off = 0;
  p->off_status = off;
  off += 256;
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
    LUB_TRY(launch_diag_factor(st, dg, lda, w, ofs + p0, first_bad));
    const int64_t rest = updm - (p0 + w);
    if (rest > 0) {
      LUB_TRY(launch_lpanel(st, dg + w, lda, dg, rest, w));
      LUB_TRY(launch_upanel(st, dg + (int64_t)w * lda, lda, dg, rest, w));
    }
    if (p0 + w < in) {
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
                           int64_t lda, int* first_bad) {
  const int64_t n = p.n, nb = p.nb;
  for (int64_t ofs = 0; ofs < n; ofs += nb) {
    const int64_t in = std::min(n - ofs, nb);
    const int64_t updm = n - ofs;
    LUB_TRY(factor_block(p, st, a, lda, ofs, in, updm, first_bad));
    const int64_t ofst = ofs + nb;
    const int64_t tn = n - ofst;
    if (tn > 0) {
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
  lu_status s = launch_fill_int(st, first_bad, kNoBadPivot, 1);
  if (s == LU_SUCCESS && n > 0)
    s = rl_factor(p, st, static_cast<float*>(d_a), lda, first_bad);
  if (s == LU_SUCCESS) s = launch_finalize_info(st, first_bad, d_info);
  if (s == LU_SUCCESS && d_a_lowp != nullptr && n > 0)
    s = launch_convert(st, m, n, d_a, LU_F32, lda, d_a_lowp, LU_F16, ld_lowp, 0);
  if (owned) cudaFreeAsync(ws, st);
  return s;
}

lu_status gemm_update(lu_compute compute, cudaStream_t st, int64_t m, int64_t n,
                      int64_t k, double alpha, const float* a, int64_t lda,
                      const float* b, int64_t ldb, double beta, float* c,
                      int64_t ldc, void* workspace, size_t ws_bytes) {
  (void)workspace;
  (void)ws_bytes;
  if (compute == LU_COMPUTE_FP32)
    return launch_sgemm_update(st, m, n, k, (float)alpha, a, lda, b, ldb,
                               (float)beta, c, ldc, false);
  return LU_ERR_UNSUPPORTED;
}

}  // namespace lub
