/*
 * remifa_shim.hxx -- header-only C++ drop-in for the lu_nopiv API of
 * flipflapflop/remifa, implemented on the C ABI of liblu_b200.so.
 *
 * A C++ caller of the reference keeps its code: the templates
 * remifa::lu_nopiv_rl / lu_nopiv_ll, the non-template lu_nopiv_ll_* wrappers,
 * remifa::lu_nopiv_panel, remifa::convert, remifa::gemmex, remifa::align_lda
 * and the tags (compute_type, CublasImpl, CutlassImpl, CutlassSplitKImpl, TC,
 * FP) have the reference's names, template parameters and signatures
 * (src/lu_nopiv.hxx:44-63, src/lu_nopiv_ll.hxx:41-66 and 586-793,
 * src/lu_nopiv.cuh:12-19, src/convert.cuh:17-18, src/gemm.cuh:17-40,
 * src/utils.hxx:18-24, 48-62).  The headers in include/remifa/ carry the
 * reference's file names and include this one, so `-I include/remifa
 * -I include` replaces `-I src` of the reference; link liblu_b200.so and
 * cuBLAS (for the handle type).
 *
 * Behaviour kept from the reference:
 *   - the cublasHandle_t is used only to fetch the stream (cublasGetStream,
 *     src/lu_nopiv.hxx:94); no cuBLAS routine computes anything;
 *   - lu_nopiv_rl / lu_nopiv_ll return after cudaStreamSynchronize
 *     (src/lu_nopiv.hxx:200, src/lu_nopiv_ll.hxx:575);
 *   - CUDA / library failures throw std::runtime_error, bad or unsupported
 *     arguments std::invalid_argument (src/errchk.hxx:18-43,
 *     src/lu_nopiv_inner_ll.hxx:67-105), including the reference's check that
 *     fp32 storage with TC32 outer updates gets an fp16 copy buffer
 *     (src/lu_nopiv.hxx:80-83, src/lu_nopiv_ll.hxx:131-135).  Where the
 *     reference calls std::exit(0) on an unsupported compute type
 *     (src/lu_nopiv_ll.hxx:78-88) this throws std::invalid_argument.
 * Differences (all documented in lu_b200.h):
 *   - *d_info is 0 on success, or the 1-based column of the first zero /
 *     non-finite pivot (the reference writes n);
 *   - CUTLASS and CUTLASS split-K implementation tags select the same
 *     tcgen05 kernels as cuBLAS (the library has one GEMM implementation);
 *     `slices` and `workspace` are accepted and ignored;
 *   - inner updates (I) always run in fp32 (K = 8 rank updates are far
 *     below a tensor-core tile), which is at least as accurate as the
 *     reference's TC32 / FP16 / TC16 inner updates; outer TC16 / FP16 updates
 *     of fp16 matrices run on the tensor cores with fp32 accumulation and one
 *     rounding to fp16;
 *   - the fp16 copy buffer receives the fp16 copy of the final factors.
 */
#ifndef REMIFA_SHIM_HXX
#define REMIFA_SHIM_HXX

#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <type_traits>

#include <cublas_v2.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "lu_b200.h"

namespace remifa {

using half = __half;

/* src/utils.hxx:18-24 (same values as lu_compute 0..3) */
enum compute_type { FP32 = LU_COMPUTE_FP32, FP16 = LU_COMPUTE_FP16,
                    TC32 = LU_COMPUTE_TC32, TC16 = LU_COMPUTE_TC16 };

/* src/gemm.cuh:17-22 */
struct CublasImpl;
struct CutlassImpl;
struct CutlassSplitKImpl;
struct TC;
struct FP;

namespace shim {

inline std::string message(lu_status s, const std::string& ctx) {
  std::string m = "[" + ctx + "] " + lu_status_string(s);
  const char* e = lu_last_error();
  if (e && *e) m += std::string(" (") + e + ")";
  return m;
}

/* Status -> the reference's exception types. */
inline void check(lu_status s, const std::string& ctx) {
  switch (s) {
    case LU_SUCCESS:
      return;
    case LU_ERR_INVALID_ARG:
    case LU_ERR_UNSUPPORTED:
    case LU_ERR_WORKSPACE:
      throw std::invalid_argument(message(s, ctx));
    default:
      throw std::runtime_error(message(s, ctx));
  }
}

inline void cuda_check(cudaError_t e, const std::string& ctx) {
  if (e != cudaSuccess)
    throw std::runtime_error("[" + ctx + "][CUDA error] (" +
                             std::string(cudaGetErrorString(e)) + ")");
}

inline cudaStream_t stream_of(cublasHandle_t h, const std::string& ctx) {
  cudaStream_t st = nullptr;
  const cublasStatus_t s = cublasGetStream(h, &st);
  if (s != CUBLAS_STATUS_SUCCESS)
    throw std::runtime_error("[" + ctx + "][cuBLAS error] (" + std::to_string((int)s) + ")");
  return st;
}

inline cudaStream_t stream_of(cudaStream_t st, const std::string&) { return st; }

template <typename T> struct dtype;
template <> struct dtype<float> { static constexpr lu_dtype value = LU_F32; };
template <> struct dtype<half> { static constexpr lu_dtype value = LU_F16; };
template <> struct dtype<double> { static constexpr lu_dtype value = LU_F64; };

template <typename T>
inline lu_stream_t as_lu(T st) { return reinterpret_cast<lu_stream_t>(st); }

}  // namespace shim

/* src/utils.hxx:48-62: lda rounded up to a multiple of 64 bytes. */
template <typename T>
size_t align_lda(size_t lda) {
  constexpr int align = 64;
  static_assert(align % sizeof(T) == 0, "Can only align if T divides align");
  constexpr size_t t = align / sizeof(T);
  return t * ((lda - 1) / t + 1);
}

/* remifa::lu_nopiv_rl (src/lu_nopiv.hxx:44-63) -> lu_nopiv_rl_c. */
template <typename T, compute_type I = FP32, compute_type O = FP32, int ib = 8,
          bool use_cutlass = false, typename CpyType = half>
void lu_nopiv_rl(const cublasHandle_t cuhandle, std::int64_t m, std::int64_t n,
                 std::int64_t nb, T* const d_a, std::int64_t ldda, int* d_info,
                 CpyType* d_a_cpy = nullptr, std::int64_t ld_a_cpy = -1) {
  const std::string ctx = "lu_nopiv_rl";
  if (std::is_same<T, float>::value && O == TC32 && d_a_cpy == nullptr)
    throw std::invalid_argument("A fp16 buffer should be provided");
  const cudaStream_t st = shim::stream_of(cuhandle, ctx);
  lu_opts o;
  lu_opts_default(&o);
  o.nb = nb;
  o.ib = ib;
  o.inner_update = I;
  o.outer_update = O;
  void* cpy = std::is_same<CpyType, half>::value ? (void*)d_a_cpy : nullptr;
  shim::check(lu_nopiv_rl_c(&o, shim::as_lu(st), m, n, d_a, shim::dtype<T>::value, ldda,
                            d_info, cpy, cpy ? ld_a_cpy : 0, nullptr, 0),
              ctx);
  shim::cuda_check(cudaStreamSynchronize(st), ctx);
}

/* remifa::lu_nopiv_ll (src/lu_nopiv_ll.hxx:41-66) -> lu_nopiv_ll_c.  OP (the
 * outer panel precision) float with fp16 storage keeps the block column /
 * row update in fp32 until the panel is factored (opts.panel_fp32). */
template <typename T, compute_type I = FP32, compute_type O = FP32, std::int64_t ib = 8,
          typename OP = T, typename IP = T, typename OF = T, typename IF = OF,
          typename GemmImpl = CublasImpl, typename CpyType = half>
void lu_nopiv_ll(const cublasHandle_t cuhandle, std::int64_t m, std::int64_t n,
                 std::int64_t nb, T* const d_a, std::int64_t ldda, int* d_info,
                 int slices = 0, uint8_t* workspace = nullptr, CpyType* d_a_cpy = nullptr,
                 std::int64_t ld_a_cpy = -1) {
  (void)slices;
  (void)workspace;
  const std::string ctx = "lu_nopiv_ll";
  // src/lu_nopiv_ll.hxx:78-88 (the reference exits here)
  if ((O == TC16 || O == FP16) && !std::is_same<OP, half>::value)
    throw std::invalid_argument("[lu_nopiv_ll] Update compute type NOT supported");
  constexpr bool w32 = std::is_same<T, float>::value;
  if (w32 && O == TC32 && d_a_cpy == nullptr)
    throw std::invalid_argument("A fp16 buffer should be provided");
  // the inner factorization's checks (src/lu_nopiv_inner_ll.hxx:67-105)
  if (m <= 0) throw std::invalid_argument("Given number of rows invalid: m = " + std::to_string(m));
  if (n <= 0)
    throw std::invalid_argument("Given number of columns invalid: n = " + std::to_string(n));
  if (w32 && I == TC32 && (d_a_cpy == nullptr || ld_a_cpy <= 0))
    throw std::invalid_argument(
        "A fp16 buffer should be provided to this routine when W=fp32 and U=TC32");
  if (w32 && I == TC16) throw std::invalid_argument("TC16 compute type unavailable with W=fp32");
  if (w32 && !(std::is_same<IP, float>::value && std::is_same<IF, float>::value))
    throw std::invalid_argument("Only fp32 factor type available with W=fp32");
  if (!w32 && I == FP32)
    throw std::invalid_argument("FP32 compute type unavailable with W=fp16");
  const cudaStream_t st = shim::stream_of(cuhandle, ctx);
  lu_opts o;
  lu_opts_default(&o);
  o.nb = nb;
  o.ib = (int32_t)ib;
  o.inner_update = I;
  o.outer_update = O;
  o.panel_fp32 = std::is_same<T, half>::value && std::is_same<OP, float>::value ? 1 : 0;
  // fp16 storage: the fp16 matrix is its own low-precision copy
  void* cpy = std::is_same<T, float>::value && std::is_same<CpyType, half>::value &&
                      (void*)d_a_cpy != (void*)d_a
                  ? (void*)d_a_cpy
                  : nullptr;
  shim::check(lu_nopiv_ll_c(&o, shim::as_lu(st), m, n, d_a, shim::dtype<T>::value, ldda,
                            d_info, cpy, cpy ? ld_a_cpy : 0, nullptr, 0),
              ctx);
  shim::cuda_check(cudaStreamSynchronize(st), ctx);
}

/* remifa::lu_nopiv_panel<T, ib> (src/lu_nopiv.cuh:12-19) -> lu_panel_c. */
template <typename T, int ib = 8>
void lu_nopiv_panel(const cudaStream_t stream, int m, int n, T const* const d, int ldd,
                    T* l, int ldl, T* u, int ldu, int* stat) {
  static_assert(ib == 8, "lu_panel_c factors 8-column tiles");
  shim::check(lu_panel_c(shim::as_lu(stream), shim::dtype<T>::value, m, n, d, ldd, l, ldl,
                         u, ldu, stat),
              "lu_nopiv_panel");
}

/* remifa::convert<TA, TAO> (src/convert.cuh:17-18) -> lu_convert_c. */
template <typename TA, typename TAO>
void convert(cudaStream_t const stream, int m, int n, TA* const a, int lda,
             TAO* const aout, int ldaout) {
  shim::check(lu_convert_c(shim::as_lu(stream), m, n, a, shim::dtype<TA>::value, lda, aout,
                           shim::dtype<TAO>::value, ldaout, 0),
              "convert");
}

/* remifa::gemmex (src/gemm.cuh:24-40) -> lu_gemm_update_ex_c:
 * c = alpha a b + beta c.  Op TC / FP with fp16 operands select the
 * tensor-core kinds TC32 (fp32 accumulator type) or TC16 (fp16); fp32
 * operands with Op FP the SIMT fp32 update.  The queue is a cuBLAS handle
 * (CublasImpl) or a stream (CUTLASS tags), as in the reference. */
template <typename GemmImpl = CublasImpl, typename Op = FP, typename AccType,
          typename InType, typename OutType = InType, typename StreamType = cudaStream_t>
void gemmex(StreamType const stream, int m, int n, int k, AccType alpha, InType const* a,
            int lda, InType const* b, int ldb, AccType beta, OutType* c, int ldc,
            int slices = 0, uint8_t* workspace = nullptr) {
  (void)slices;
  (void)workspace;
  const std::string ctx = "gemmex";
  constexpr bool tc = std::is_same<Op, TC>::value;
  constexpr bool acc16 = std::is_same<AccType, half>::value;
  const lu_compute compute =
      std::is_same<InType, float>::value && !tc ? LU_COMPUTE_FP32
      : acc16                                   ? (tc ? LU_COMPUTE_TC16 : LU_COMPUTE_FP16)
                                                : LU_COMPUTE_TC32;
  const cudaStream_t st = shim::stream_of(stream, ctx);
  shim::check(lu_gemm_update_ex_c(shim::as_lu(st), compute, m, n, k, (double)(float)alpha,
                                  a, shim::dtype<InType>::value, lda, b,
                                  shim::dtype<InType>::value, ldb, (double)(float)beta, c,
                                  shim::dtype<OutType>::value, ldc, nullptr, 0),
              ctx);
}

/* ---- the non-template wrappers of src/lu_nopiv_ll.hxx:586-793 ---------- */

#define REMIFA_SHIM_LL_F32(NAME, I, O)                                                  \
  inline void NAME(const cublasHandle_t h, int m, int n, int nb, float* const d_a,    \
                   int ldda, int* d_info) {                                           \
    lu_nopiv_ll<float, I, O, 8>(h, m, n, nb, d_a, ldda, d_info);                      \
  }
#define REMIFA_SHIM_LL_F32_SPLITK(NAME, I, O)                                           \
  inline void NAME(const cublasHandle_t h, int m, int n, int nb, float* const d_a,    \
                   int ldda, int* d_info, int slices, uint8_t* workspace) {           \
    lu_nopiv_ll<float, I, O, 8>(h, m, n, nb, d_a, ldda, d_info, slices, workspace);   \
  }
#define REMIFA_SHIM_LL_F32_TC(NAME, I)                                                  \
  inline void NAME(const cublasHandle_t h, int m, int n, int nb, float* const d_a,    \
                   int ldda, int* d_info, half* d_a_f16, int ld_a_f16) {              \
    lu_nopiv_ll<float, I, TC32, 8>(h, m, n, nb, d_a, ldda, d_info, 0, nullptr,        \
                                   d_a_f16, ld_a_f16);                                \
  }
#define REMIFA_SHIM_LL_F32_TC_SPLITK(NAME, I)                                           \
  inline void NAME(const cublasHandle_t h, int m, int n, int nb, float* const d_a,    \
                   int ldda, int* d_info, int slices, uint8_t* workspace,             \
                   half* d_a_f16, int ld_a_f16) {                                     \
    lu_nopiv_ll<float, I, TC32, 8>(h, m, n, nb, d_a, ldda, d_info, slices, workspace, \
                                   d_a_f16, ld_a_f16);                                \
  }
#define REMIFA_SHIM_LL_F16(NAME, I, O, OP)                                              \
  inline void NAME(const cublasHandle_t h, int m, int n, int nb, half* const d_a,     \
                   int ldda, int* d_info) {                                           \
    lu_nopiv_ll<half, I, O, 8, OP>(h, m, n, nb, d_a, ldda, d_info);                   \
  }
#define REMIFA_SHIM_LL_F16_SPLITK(NAME, I, O, OP)                                       \
  inline void NAME(const cublasHandle_t h, int m, int n, int nb, half* const d_a,     \
                   int ldda, int* d_info, int slices, uint8_t* workspace) {           \
    lu_nopiv_ll<half, I, O, 8, OP>(h, m, n, nb, d_a, ldda, d_info, slices, workspace); \
  }

/* W = fp32 (src/lu_nopiv_ll.cxx:14-185) */
REMIFA_SHIM_LL_F32(lu_nopiv_ll_f32, FP32, FP32)
REMIFA_SHIM_LL_F32(lu_nopiv_ll_cutlass_f32, FP32, FP32)
REMIFA_SHIM_LL_F32_SPLITK(lu_nopiv_ll_cutlass_splitk_f32, FP32, FP32)
REMIFA_SHIM_LL_F32_TC(lu_nopiv_ll_f32_fp32xtc32, FP32)
REMIFA_SHIM_LL_F32_TC(lu_nopiv_ll_cutlass_f32_fp32xtc32, FP32)
REMIFA_SHIM_LL_F32_TC_SPLITK(lu_nopiv_ll_cutlass_splitk_f32_fp32xtc32, FP32)
REMIFA_SHIM_LL_F32_TC(lu_nopiv_ll_f32_tc32xtc32, TC32)
REMIFA_SHIM_LL_F32_TC(lu_nopiv_ll_cutlass_f32_tc32xtc32, TC32)
REMIFA_SHIM_LL_F32_TC_SPLITK(lu_nopiv_ll_cutlass_splitk_f32_tc32xtc32, TC32)
/* W = fp16 (src/lu_nopiv_ll.cxx:191-670) */
REMIFA_SHIM_LL_F16(lu_nopiv_ll_f16, FP16, FP16, half)
REMIFA_SHIM_LL_F16(lu_nopiv_ll_cutlass_f16, FP16, FP16, half)
REMIFA_SHIM_LL_F16_SPLITK(lu_nopiv_ll_cutlass_splitk_f16, FP16, FP16, half)
REMIFA_SHIM_LL_F16(lu_nopiv_ll_f16_f16xtc16, FP16, TC16, half)
REMIFA_SHIM_LL_F16(lu_nopiv_ll_cutlass_f16_f16xtc16, FP16, TC16, half)
REMIFA_SHIM_LL_F16_SPLITK(lu_nopiv_ll_cutlass_splitk_f16_f16xtc16, FP16, TC16, half)
REMIFA_SHIM_LL_F16(lu_nopiv_ll_f16_tc16xtc16, TC16, TC16, half)
REMIFA_SHIM_LL_F16(lu_nopiv_ll_cutlass_f16_tc16xtc16, TC16, TC16, half)
REMIFA_SHIM_LL_F16(lu_nopiv_ll_f16_tc32xtc32, TC32, TC32, half)
REMIFA_SHIM_LL_F16(lu_nopiv_ll_cutlass_f16_tc32xtc32, TC32, TC32, half)
REMIFA_SHIM_LL_F16_SPLITK(lu_nopiv_ll_cutlass_splitk_f16_tc32xtc32, TC32, TC32, half)
REMIFA_SHIM_LL_F16(lu_nopiv_ll_f16_f16xtc32, FP16, TC32, half)
REMIFA_SHIM_LL_F16(lu_nopiv_ll_cutlass_f16_f16xtc32, FP16, TC32, half)
REMIFA_SHIM_LL_F16_SPLITK(lu_nopiv_ll_cutlass_splitk_f16_f16xtc32, FP16, TC32, half)
REMIFA_SHIM_LL_F16(lu_nopiv_ll_f16_f16xtc32_fp32, FP16, TC32, float)
REMIFA_SHIM_LL_F16(lu_nopiv_ll_cutlass_f16_f16xtc32_fp32, FP16, TC32, float)
REMIFA_SHIM_LL_F16_SPLITK(lu_nopiv_ll_cutlass_splitk_f16_f16xtc32_fp32, FP16, TC32, float)
REMIFA_SHIM_LL_F16(lu_nopiv_ll_f16_f32xt32, FP32, TC32, float)
REMIFA_SHIM_LL_F16(lu_nopiv_ll_cutlass_f16_f32xtc32, FP32, TC32, float)
REMIFA_SHIM_LL_F16_SPLITK(lu_nopiv_ll_cutlass_splitk_f16_f32xtc32, FP32, TC32, float)
REMIFA_SHIM_LL_F16(lu_nopiv_ll_f16_tc32xtc32_fp16xfp32_fp16xfp32, TC32, TC32, half)
REMIFA_SHIM_LL_F16(lu_nopiv_ll_cutlass_f16_tc32xtc32_fp16xfp32_fp16xfp32, TC32, TC32, half)
REMIFA_SHIM_LL_F16_SPLITK(lu_nopiv_ll_cutlass_splitk_f16_tc32xtc32_fp16xfp32_fp16xfp32,
                          TC32, TC32, half)
REMIFA_SHIM_LL_F16(lu_nopiv_ll_f16_tc32xtc32_fp32xfp32_fp32xfp32, TC32, TC32, float)
REMIFA_SHIM_LL_F16(lu_nopiv_ll_cutlass_f16_tc32xtc32_fp32xfp32_fp32xfp32, TC32, TC32, float)
REMIFA_SHIM_LL_F16_SPLITK(lu_nopiv_ll_cutlass_splitk_f16_tc32xtc32_fp32xfp32_fp32xfp32,
                          TC32, TC32, float)

#undef REMIFA_SHIM_LL_F32
#undef REMIFA_SHIM_LL_F32_SPLITK
#undef REMIFA_SHIM_LL_F32_TC
#undef REMIFA_SHIM_LL_F32_TC_SPLITK
#undef REMIFA_SHIM_LL_F16
#undef REMIFA_SHIM_LL_F16_SPLITK

}  // namespace remifa

#endif  // REMIFA_SHIM_HXX
