// C-ABI entry points and the host-side factorization drivers.
//
// Host drivers are ordinary C++: they enqueue the panel kernels and the
// update kernels on the caller's stream (plus an internal look-ahead stream
// when enabled) and return without synchronising, unlike the reference,
// which synchronises and frees its workspace at the end of every call
// (src/lu_nopiv.hxx:200-205).
#include "common.cuh"
#include "kernels.cuh"
#include "driver.cuh"
#include "rowsolve.cuh"

#include <algorithm>
#include <cstring>

namespace lub {
const char* last_error_message();
}

using namespace lub;

extern "C" {

void lu_opts_default(lu_opts* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->nb = 256;
  o->ib = 8;
  o->inner_update = LU_COMPUTE_FP32;
  o->outer_update = LU_COMPUTE_FP32;
  o->variant = LU_RIGHT_LOOKING;
  o->lookahead = 1;
  o->diag_width = 0;
}

int lu_abi_version(void) { return LU_B200_ABI_VERSION; }

const char* lu_status_string(lu_status s) {
  switch (s) {
    case LU_SUCCESS: return "success";
    case LU_ERR_INVALID_ARG: return "invalid argument";
    case LU_ERR_CUDA: return "CUDA error";
    case LU_ERR_ALLOC: return "device allocation failed";
    case LU_ERR_UNSUPPORTED: return "unsupported combination";
    case LU_ERR_WORKSPACE: return "workspace too small";
    case LU_ERR_NOT_CONVERGED: return "iterative refinement did not converge";
    case LU_ERR_TIMEOUT: return "device wait timed out";
    case LU_ERR_NO_DEVICE: return "no sm_100 device";
  }
  return "unknown status";
}

const char* lu_last_error(void) { return last_error_message(); }

lu_status lu_workspace_size(const lu_opts* opts, int64_t m, int64_t n,
                            lu_dtype dtype_a, size_t* bytes) {
  if (!bytes) return LU_ERR_INVALID_ARG;
  lu_opts o;
  if (opts) o = *opts; else lu_opts_default(&o);
  Plan p;
  LUB_TRY(make_plan(o, m, n, dtype_a, &p));
  *bytes = p.ws_bytes;
  return LU_SUCCESS;
}

lu_status lu_nopiv_rl_c(const lu_opts* opts, lu_stream_t stream, int64_t m,
                        int64_t n, void* d_a, lu_dtype dtype_a, int64_t lda,
                        int* d_info, void* d_a_lowp, int64_t ld_lowp,
                        void* workspace, size_t ws_bytes) {
  lu_opts o;
  if (opts) o = *opts; else lu_opts_default(&o);
  o.variant = LU_RIGHT_LOOKING;
  return factorize(o, (cudaStream_t)stream, m, n, d_a, dtype_a, lda, d_info,
                   d_a_lowp, ld_lowp, workspace, ws_bytes);
}

lu_status lu_nopiv_rl_host_c(const lu_opts* opts, lu_stream_t stream, int64_t n,
                             float* h_a, int64_t lda, float* d_a, int64_t ldda,
                             int* d_info, void* workspace, size_t ws_bytes) {
  lu_opts o;
  if (opts) o = *opts; else lu_opts_default(&o);
  o.variant = LU_RIGHT_LOOKING;
  return factorize_host(o, (cudaStream_t)stream, n, h_a, lda, d_a, ldda, d_info,
                        workspace, ws_bytes);
}

lu_status lu_nopiv_ll_c(const lu_opts* opts, lu_stream_t stream, int64_t m,
                        int64_t n, void* d_a, lu_dtype dtype_a, int64_t lda,
                        int* d_info, void* d_a_lowp, int64_t ld_lowp,
                        void* workspace, size_t ws_bytes) {
  lu_opts o;
  if (opts) o = *opts; else lu_opts_default(&o);
  o.variant = LU_LEFT_LOOKING;
  return factorize(o, (cudaStream_t)stream, m, n, d_a, dtype_a, lda, d_info,
                   d_a_lowp, ld_lowp, workspace, ws_bytes);
}

lu_status lu_panel_c(lu_stream_t stream, lu_dtype dtype, int64_t m, int64_t n,
                     const void* d, int64_t ldd, void* l, int64_t ldl, void* u,
                     int64_t ldu, int* stat) {
  if (dtype != LU_F32 && dtype != LU_F16) return LU_ERR_UNSUPPORTED;
  if (n <= 0 || n > 8 || m < n || !d || !l || !u) return LU_ERR_INVALID_ARG;
  if (ldd < n || ldl < m || ldu < n) return LU_ERR_INVALID_ARG;
  LUB_TRY(check_device());
  if (dtype == LU_F16)
    return launch_ref_panel_f16((cudaStream_t)stream, m, (int)n, (const __half*)d, ldd,
                                (__half*)l, ldl, (__half*)u, ldu, stat);
  return launch_ref_panel((cudaStream_t)stream, m, (int)n, (const float*)d, ldd,
                          (float*)l, ldl, (float*)u, ldu, stat);
}

lu_status lu_convert_c(lu_stream_t stream, int64_t m, int64_t n, const void* a,
                       lu_dtype type_a, int64_t lda, void* out,
                       lu_dtype type_out, int64_t ldout, int scale_log2) {
  LUB_TRY(check_device());
  return launch_convert((cudaStream_t)stream, m, n, a, type_a, lda, out,
                        type_out, ldout, scale_log2);
}

lu_status lu_gemm_update_c(lu_stream_t stream, lu_compute compute, int64_t m,
                           int64_t n, int64_t k, double alpha, const void* a,
                           int64_t lda, const void* b, int64_t ldb,
                           double beta, void* c, int64_t ldc, void* workspace,
                           size_t ws_bytes) {
  if (m < 0 || n < 0 || k < 0) return LU_ERR_INVALID_ARG;
  if (m == 0 || n == 0) return LU_SUCCESS;
  if (!a || !b || !c) return LU_ERR_INVALID_ARG;
  if (lda < std::max<int64_t>(1, m) || ldb < std::max<int64_t>(1, k) ||
      ldc < std::max<int64_t>(1, m))
    return LU_ERR_INVALID_ARG;
  LUB_TRY(check_device());
  return gemm_update(compute, (cudaStream_t)stream, m, n, k, alpha,
                     (const float*)a, lda, (const float*)b, ldb, beta,
                     (float*)c, ldc, workspace, ws_bytes);
}

lu_status lu_gemm_update_ex_c(lu_stream_t stream, lu_compute compute, int64_t m,
                              int64_t n, int64_t k, double alpha, const void* a,
                              lu_dtype type_a, int64_t lda, const void* b, lu_dtype type_b,
                              int64_t ldb, double beta, void* c, lu_dtype type_c,
                              int64_t ldc, void* workspace, size_t ws_bytes) {
  if (m < 0 || n < 0 || k < 0) return LU_ERR_INVALID_ARG;
  if (m == 0 || n == 0) return LU_SUCCESS;
  if (!a || !b || !c) return LU_ERR_INVALID_ARG;
  if (lda < std::max<int64_t>(1, m) || ldb < std::max<int64_t>(1, k) ||
      ldc < std::max<int64_t>(1, m))
    return LU_ERR_INVALID_ARG;
  LUB_TRY(check_device());
  return gemm_update_ex(compute, (cudaStream_t)stream, m, n, k, alpha, a, type_a, lda, b,
                        type_b, ldb, beta, c, type_c, ldc, workspace, ws_bytes);
}

lu_status lu_gen_matrix_c(lu_stream_t stream, int64_t n, float* d_a,
                          int64_t lda, uint64_t seed, int kind, double alpha,
                          int kscale, double gamma_bits) {
  LUB_TRY(check_device());
  return launch_gen_matrix((cudaStream_t)stream, n, d_a, lda, seed, kind,
                           alpha, kscale, gamma_bits);
}

lu_status lu_catchup_row_step_c(lu_stream_t stream, int fused, int bf16, int64_t in, int64_t nc,
                                int64_t coff, int64_t kl, float* d_a, int64_t lda,
                                const void* d_la, int64_t lda_k, const void* d_xb, void* d_xo,
                                int64_t ldx, const float* d_part, int64_t slab, int64_t ldp,
                                int nslabs, int* d_err) {
  if (in <= 0 || nc < 0 || coff < in || kl < 0 || !d_a || !d_xo || !d_err || nslabs < 0)
    return LU_ERR_INVALID_ARG;
  if (nslabs > 0 && (!d_part || ldp != (in + 3) / 4 * 4 || slab < ldp * nc || slab % 4 != 0))
    return LU_ERR_INVALID_ARG;
  if (lda < in || ldx < in || (kl > 0 && (!d_la || !d_xb || lda_k < kl || ldx < kl)))
    return LU_ERR_INVALID_ARG;
  if (fused && !rowsolve_supported(in, kl, ldx)) return LU_ERR_UNSUPPORTED;
  if (!fused && (in % 8 != 0 || kl % 8 != 0 || ldx % 8 != 0 || lda_k % 8 != 0))
    return LU_ERR_UNSUPPORTED;
  LUB_TRY(check_device());
  EarlyPart ep;
  ep.part = d_part;
  ep.slab = slab;
  ep.ldp = ldp;
  ep.ns = nslabs;
  return catchup_row_step((cudaStream_t)stream, fused != 0, bf16 != 0, d_a, lda, in, coff, nc,
                          kl, d_la, lda_k, d_xb, d_xo, ldx, 128, d_err, ep);
}

}  // extern "C"
