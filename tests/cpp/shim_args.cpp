// Argument errors through the C++ drop-in (include/remifa_shim.hxx), with
// no device needed: each must surface as the exception type the reference
// throws.  Also pins, at compile time, every lu_nopiv_ll_* wrapper to the
// signature the reference declares (src/lu_nopiv_ll.hxx:586-793).
// Exit status 0 when every check holds; a failing check prints its line.
#include <cstdio>
#include <stdexcept>

#include "lu_nopiv.hxx"
#include "lu_nopiv_ll.hxx"
#include "lu_nopiv.cuh"
#include "convert.cuh"
#include "gemm.cuh"
#include "utils.hxx"

using remifa::half;

static int failures = 0;

template <typename E, typename F>
static void expect(F&& f, int line) {
  try {
    f();
  } catch (const E&) {
    return;
  } catch (const std::exception& e) {
    std::printf("line %d: wrong exception: %s\n", line, e.what());
    ++failures;
    return;
  }
  std::printf("line %d: no exception\n", line);
  ++failures;
}
#define EXPECT_INVALID(expr) expect<std::invalid_argument>([&] { expr; }, __LINE__)
#define EXPECT_RUNTIME(expr) expect<std::runtime_error>([&] { expr; }, __LINE__)

using LlF32 = void (*)(const cublasHandle_t, int, int, int, float* const, int, int*);
using LlF32Sk = void (*)(const cublasHandle_t, int, int, int, float* const, int, int*, int,
                         uint8_t*);
using LlF32Tc = void (*)(const cublasHandle_t, int, int, int, float* const, int, int*, half*,
                         int);
using LlF32TcSk = void (*)(const cublasHandle_t, int, int, int, float* const, int, int*, int,
                           uint8_t*, half*, int);
using LlF16 = void (*)(const cublasHandle_t, int, int, int, half* const, int, int*);
using LlF16Sk = void (*)(const cublasHandle_t, int, int, int, half* const, int, int*, int,
                         uint8_t*);

int main() {
  // every wrapper of the reference header, with its exact type
  LlF32 f32[] = {remifa::lu_nopiv_ll_f32, remifa::lu_nopiv_ll_cutlass_f32};
  LlF32Sk f32sk[] = {remifa::lu_nopiv_ll_cutlass_splitk_f32};
  LlF32Tc f32tc[] = {remifa::lu_nopiv_ll_f32_fp32xtc32, remifa::lu_nopiv_ll_cutlass_f32_fp32xtc32,
                     remifa::lu_nopiv_ll_f32_tc32xtc32, remifa::lu_nopiv_ll_cutlass_f32_tc32xtc32};
  LlF32TcSk f32tcsk[] = {remifa::lu_nopiv_ll_cutlass_splitk_f32_fp32xtc32,
                         remifa::lu_nopiv_ll_cutlass_splitk_f32_tc32xtc32};
  LlF16 f16[] = {remifa::lu_nopiv_ll_f16,
                 remifa::lu_nopiv_ll_cutlass_f16,
                 remifa::lu_nopiv_ll_f16_f16xtc16,
                 remifa::lu_nopiv_ll_cutlass_f16_f16xtc16,
                 remifa::lu_nopiv_ll_f16_tc16xtc16,
                 remifa::lu_nopiv_ll_cutlass_f16_tc16xtc16,
                 remifa::lu_nopiv_ll_f16_tc32xtc32,
                 remifa::lu_nopiv_ll_cutlass_f16_tc32xtc32,
                 remifa::lu_nopiv_ll_f16_f16xtc32,
                 remifa::lu_nopiv_ll_cutlass_f16_f16xtc32,
                 remifa::lu_nopiv_ll_f16_f16xtc32_fp32,
                 remifa::lu_nopiv_ll_cutlass_f16_f16xtc32_fp32,
                 remifa::lu_nopiv_ll_f16_f32xt32,
                 remifa::lu_nopiv_ll_cutlass_f16_f32xtc32,
                 remifa::lu_nopiv_ll_f16_tc32xtc32_fp16xfp32_fp16xfp32,
                 remifa::lu_nopiv_ll_cutlass_f16_tc32xtc32_fp16xfp32_fp16xfp32,
                 remifa::lu_nopiv_ll_f16_tc32xtc32_fp32xfp32_fp32xfp32,
                 remifa::lu_nopiv_ll_cutlass_f16_tc32xtc32_fp32xfp32_fp32xfp32};
  LlF16Sk f16sk[] = {remifa::lu_nopiv_ll_cutlass_splitk_f16,
                     remifa::lu_nopiv_ll_cutlass_splitk_f16_f16xtc16,
                     remifa::lu_nopiv_ll_cutlass_splitk_f16_tc32xtc32,
                     remifa::lu_nopiv_ll_cutlass_splitk_f16_f16xtc32,
                     remifa::lu_nopiv_ll_cutlass_splitk_f16_f16xtc32_fp32,
                     remifa::lu_nopiv_ll_cutlass_splitk_f16_f32xtc32,
                     remifa::lu_nopiv_ll_cutlass_splitk_f16_tc32xtc32_fp16xfp32_fp16xfp32,
                     remifa::lu_nopiv_ll_cutlass_splitk_f16_tc32xtc32_fp32xfp32_fp32xfp32};
  const int nwrappers = sizeof(f32) / sizeof(f32[0]) + sizeof(f32sk) / sizeof(f32sk[0]) +
                        sizeof(f32tc) / sizeof(f32tc[0]) + sizeof(f32tcsk) / sizeof(f32tcsk[0]) +
                        sizeof(f16) / sizeof(f16[0]) + sizeof(f16sk) / sizeof(f16sk[0]);

  cublasHandle_t h = nullptr;  // never reached by the checks below
  float* a = reinterpret_cast<float*>(256);
  half* a16 = reinterpret_cast<half*>(256);
  int* info = reinterpret_cast<int*>(512);

  // fp32 storage with TC32 outer updates needs the fp16 copy buffer
  // (src/lu_nopiv.hxx:80-83)
  EXPECT_INVALID((remifa::lu_nopiv_rl<float, remifa::FP32, remifa::TC32>(h, 64, 64, 32, a, 64,
                                                                         info)));
  EXPECT_INVALID((remifa::lu_nopiv_ll<float, remifa::FP32, remifa::TC32>(h, 64, 64, 32, a, 64,
                                                                         info)));
  EXPECT_INVALID(remifa::lu_nopiv_ll_f32_tc32xtc32(h, 64, 64, 32, a, 64, info, nullptr, 64));
  // TC16 / FP16 outer updates need an fp16 panel (src/lu_nopiv_ll.hxx:78-88)
  EXPECT_INVALID((remifa::lu_nopiv_ll<float, remifa::FP32, remifa::TC16>(h, 64, 64, 32, a, 64,
                                                                         info)));
  EXPECT_INVALID((remifa::lu_nopiv_ll<float, remifa::FP32, remifa::FP16>(h, 64, 64, 32, a, 64,
                                                                         info)));
  // the inner factorization's checks (src/lu_nopiv_inner_ll.hxx:67-105)
  EXPECT_INVALID(remifa::lu_nopiv_ll_f32(h, 0, 64, 32, a, 64, info));
  EXPECT_INVALID(remifa::lu_nopiv_ll_f32(h, 64, 0, 32, a, 64, info));
  EXPECT_INVALID(remifa::lu_nopiv_ll_f16_f32xt32(h, 64, 64, 32, a16, 64, info));
  EXPECT_INVALID((remifa::lu_nopiv_ll<float, remifa::TC16, remifa::FP32>(h, 64, 64, 32, a, 64,
                                                                         info)));
  // library argument checks before any device call
  EXPECT_INVALID((remifa::lu_nopiv_panel<float, 8>(nullptr, 64, 9, a, 8, a, 64, a, 8, info)));
  EXPECT_INVALID((remifa::gemmex<remifa::CutlassImpl, remifa::FP, float, float>(
      cudaStream_t(nullptr), -1, 4, 4, -1.0f, a, 4, a, 4, 1.0f, a, 4)));
  EXPECT_INVALID((remifa::gemmex<remifa::CutlassImpl, remifa::TC, float, half, float>(
      cudaStream_t(nullptr), 8, 8, 8, -1.0f, a16, 4, a16, 8, 1.0f, a, 8)));  // lda < m
  // a cuBLAS handle that is not valid: the reference's cuBLAS error
  EXPECT_RUNTIME(remifa::lu_nopiv_ll_f32(h, 64, 64, 32, a, 64, info));

  int dev = 0;
  if (cudaGetDeviceCount(&dev) != cudaSuccess || dev == 0) {
    // valid arguments without a device: an error, never a host fallback
    EXPECT_RUNTIME((remifa::gemmex<remifa::CutlassImpl, remifa::FP, float, float>(
        cudaStream_t(nullptr), 4, 4, 4, -1.0f, a, 4, a, 4, 1.0f, a, 4)));
    EXPECT_RUNTIME((remifa::convert<float, half>(nullptr, 4, 4, a, 4, a16, 4)));
  }
  if (remifa::align_lda<float>(100) != 112 || remifa::align_lda<half>(100) != 128) {
    std::printf("align_lda\n");
    ++failures;
  }
  std::printf("wrappers %d, failures %d\n", nwrappers, failures);
  return failures == 0 ? 0 : 1;
}
