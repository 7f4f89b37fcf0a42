// TEST INFRASTRUCTURE ONLY -- never part of the product path.
//
// Thin C-ABI shim over the UNMODIFIED reference sources (compiled from the
// read-only reference tree by oracle/Makefile into oracle/_ref/).  It lets the
// GPU parity tests run the reference's own code on the same device buffers as
// the product library, so the CPU oracle (oracle/oracle.cpp) can be pinned
// against it:
//   * ref_panel_f32      -> remifa::lu_nopiv_panel<float,8>   (src/lu_nopiv.cu:364-400)
//   * ref_convert_*      -> remifa::convert<TA,TAO>           (src/convert.cu:324-360)
//   * ref_lu_nopiv_rl_*  -> remifa::lu_nopiv_rl<float,I,O,8>  (src/lu_nopiv.hxx:44-208)
//   * ref_lu_nopiv_ll_*  -> remifa::lu_nopiv_ll_* wrappers    (src/lu_nopiv_ll.cxx:14-636)
//   * ref_panel_f16      -> remifa::lu_nopiv_panel<half,8>
// Nothing here is copied from the reference; it only calls it.
#include <cstdint>
#include <stdexcept>
#include <cstdio>

#include "lu_nopiv.hxx"
#include "lu_nopiv_ll.hxx"

namespace {
cublasHandle_t make_handle(cudaStream_t stream) {
  cublasHandle_t h = nullptr;
  if (cublasCreate(&h) != CUBLAS_STATUS_SUCCESS) return nullptr;
  cublasSetStream(h, stream);
  // the reference harness selects the default math mode
  // (tests/testing_lu_gpu.hxx:1074-1075)
  cublasSetMathMode(h, CUBLAS_DEFAULT_MATH);
  return h;
}
}  // namespace

extern "C" {

int ref_panel_f32(void* stream, int m, int n, const float* d, int ldd, float* l,
                  int ldl, float* u, int ldu, int* stat) {
  remifa::lu_nopiv_panel<float, 8>((cudaStream_t)stream, m, n, d, ldd, l, ldl,
                                   u, ldu, stat);
  return (int)cudaGetLastError();
}

int ref_convert_f32_f16(void* stream, int m, int n, float* a, int lda,
                        void* out, int ldout) {
  remifa::convert<float, half>((cudaStream_t)stream, m, n, a, lda,
                               (half*)out, ldout);
  return (int)cudaGetLastError();
}

int ref_convert_f16_f32(void* stream, int m, int n, void* a, int lda,
                        float* out, int ldout) {
  remifa::convert<half, float>((cudaStream_t)stream, m, n, (half*)a, lda, out,
                               ldout);
  return (int)cudaGetLastError();
}

// outer: 0 = FP32 outer update, 1 = TC32 outer update (fp16 copy in d_cpy).
// inner: 0 = FP32 inner update, 1 = TC32 inner update.
int ref_lu_nopiv_rl_f32(void* stream, int64_t m, int64_t n, int64_t nb,
                        float* d_a, int64_t lda, int* d_info, int inner,
                        int outer, void* d_cpy, int64_t ld_cpy) {
  cublasHandle_t h = make_handle((cudaStream_t)stream);
  if (!h) return -1;
  int rc = 0;
  try {
    if (outer == 0) {
      remifa::lu_nopiv_rl<float, remifa::FP32, remifa::FP32, 8>(
          h, m, n, nb, d_a, lda, d_info);
    } else if (inner == 0) {
      remifa::lu_nopiv_rl<float, remifa::FP32, remifa::TC32, 8>(
          h, m, n, nb, d_a, lda, d_info, (half*)d_cpy, ld_cpy);
    } else {
      remifa::lu_nopiv_rl<float, remifa::TC32, remifa::TC32, 8>(
          h, m, n, nb, d_a, lda, d_info, (half*)d_cpy, ld_cpy);
    }
  } catch (std::exception& e) {
    std::fprintf(stderr, "[ref_shim] %s\n", e.what());
    rc = -2;
  }
  cublasDestroy(h);
  return rc;
}

// W=fp32, I=O=FP32 left-looking (src/lu_nopiv_ll.cxx:14-29)
int ref_lu_nopiv_ll_f32(void* stream, int m, int n, int nb, float* d_a, int lda,
                        int* d_info) {
  cublasHandle_t h = make_handle((cudaStream_t)stream);
  if (!h) return -1;
  int rc = 0;
  try {
    remifa::lu_nopiv_ll_f32(h, m, n, nb, d_a, lda, d_info);
  } catch (std::exception& e) {
    std::fprintf(stderr, "[ref_shim] %s\n", e.what());
    rc = -2;
  }
  cublasDestroy(h);
  return rc;
}

// W=fp16, I=O=TC32 left-looking (src/lu_nopiv_ll.cxx:282-296)
int ref_lu_nopiv_ll_f16_tc32(void* stream, int m, int n, int nb, void* d_a,
                             int lda, int* d_info) {
  cublasHandle_t h = make_handle((cudaStream_t)stream);
  if (!h) return -1;
  int rc = 0;
  try {
    remifa::lu_nopiv_ll_f16_tc32xtc32(h, m, n, nb, (half*)d_a, lda, d_info);
  } catch (std::exception& e) {
    std::fprintf(stderr, "[ref_shim] %s\n", e.what());
    rc = -2;
  }
  cublasDestroy(h);
  return rc;
}

// Every cuBLAS (non-CUTLASS) W = fp16 wrapper of src/lu_nopiv_ll.cxx, by
// number:
//   0 lu_nopiv_ll_f16                                   (:191, I=O=FP16)
//   1 lu_nopiv_ll_f16_tc16xtc16                         (:246, I=O=TC16)
//   2 lu_nopiv_ll_f16_tc32xtc32                         (:282, I=O=TC32)
//   3 lu_nopiv_ll_f16_f16xtc32                          (:338, I=FP16, O=TC32)
//   4 lu_nopiv_ll_f16_f16xtc32_fp32                     (:393, OP=fp32)
//   5 lu_nopiv_ll_f16_f16xtc16                          (:507, I=FP16, O=TC16)
//   6 lu_nopiv_ll_f16_tc32xtc32_fp16xfp32_fp16xfp32     (:563, IP=IF=fp32)
//   7 lu_nopiv_ll_f16_tc32xtc32_fp32xfp32_fp32xfp32     (:618, OP=OF=IP=IF=fp32)
// Returns -3 for an unknown number.
int ref_lu_nopiv_ll_f16_variant(void* stream, int variant, int m, int n, int nb,
                                void* d_a, int lda, int* d_info) {
  cublasHandle_t h = make_handle((cudaStream_t)stream);
  if (!h) return -1;
  half* a = (half*)d_a;
  int rc = 0;
  try {
    switch (variant) {
      case 0: remifa::lu_nopiv_ll_f16(h, m, n, nb, a, lda, d_info); break;
      case 1: remifa::lu_nopiv_ll_f16_tc16xtc16(h, m, n, nb, a, lda, d_info); break;
      case 2: remifa::lu_nopiv_ll_f16_tc32xtc32(h, m, n, nb, a, lda, d_info); break;
      case 3: remifa::lu_nopiv_ll_f16_f16xtc32(h, m, n, nb, a, lda, d_info); break;
      case 4: remifa::lu_nopiv_ll_f16_f16xtc32_fp32(h, m, n, nb, a, lda, d_info); break;
      case 5: remifa::lu_nopiv_ll_f16_f16xtc16(h, m, n, nb, a, lda, d_info); break;
      case 6:
        remifa::lu_nopiv_ll_f16_tc32xtc32_fp16xfp32_fp16xfp32(h, m, n, nb, a, lda, d_info);
        break;
      case 7:
        remifa::lu_nopiv_ll_f16_tc32xtc32_fp32xfp32_fp32xfp32(h, m, n, nb, a, lda, d_info);
        break;
      default: rc = -3;
    }
  } catch (std::exception& e) {
    std::fprintf(stderr, "[ref_shim] %s\n", e.what());
    rc = -2;
  }
  cublasDestroy(h);
  return rc;
}

// W = fp32 left-looking with tensor-core outer updates, which need the fp16
// copy buffer (src/lu_nopiv_ll.cxx:74-89 fp32xtc32, :131-146 tc32xtc32).
int ref_lu_nopiv_ll_f32_tc(void* stream, int inner_tc, int m, int n, int nb,
                           float* d_a, int lda, int* d_info, void* d_cpy, int ld_cpy) {
  cublasHandle_t h = make_handle((cudaStream_t)stream);
  if (!h) return -1;
  int rc = 0;
  try {
    if (inner_tc)
      remifa::lu_nopiv_ll_f32_tc32xtc32(h, m, n, nb, d_a, lda, d_info, (half*)d_cpy, ld_cpy);
    else
      remifa::lu_nopiv_ll_f32_fp32xtc32(h, m, n, nb, d_a, lda, d_info, (half*)d_cpy, ld_cpy);
  } catch (std::exception& e) {
    std::fprintf(stderr, "[ref_shim] %s\n", e.what());
    rc = -2;
  }
  cublasDestroy(h);
  return rc;
}

// lu_nopiv_panel<half, 8> (src/lu_nopiv.cu:364-400 instantiated for half)
int ref_panel_f16(void* stream, int m, int n, const void* d, int ldd, void* l,
                  int ldl, void* u, int ldu, int* stat) {
  remifa::lu_nopiv_panel<half, 8>((cudaStream_t)stream, m, n, (const half*)d, ldd,
                                  (half*)l, ldl, (half*)u, ldu, stat);
  return (int)cudaGetLastError();
}

}  // extern "C"
