// The C++ drop-in (include/remifa_shim.hxx) on a device: every call must
// give exactly what the C ABI call it maps to gives, return with the stream
// synchronised, and report success in *d_info.  Exit status 0 on success.
#include <cstdio>
#include <cstring>
#include <vector>

#include "lu_nopiv.hxx"
#include "lu_nopiv_ll.hxx"
#include "lu_nopiv.cuh"
#include "convert.cuh"
#include "gemm.cuh"

using remifa::half;

static int failures = 0;
#define CHECK(cond)                                        \
  do {                                                     \
    if (!(cond)) {                                         \
      std::printf("line %d: %s\n", __LINE__, #cond);       \
      ++failures;                                          \
    }                                                      \
  } while (0)

template <typename T>
static bool same(const T* x, const T* y, size_t count) {
  std::vector<T> a(count), b(count);
  cudaMemcpy(a.data(), x, count * sizeof(T), cudaMemcpyDeviceToHost);
  cudaMemcpy(b.data(), y, count * sizeof(T), cudaMemcpyDeviceToHost);
  return std::memcmp(a.data(), b.data(), count * sizeof(T)) == 0;
}

static int info_of(const int* d) {
  int v = -99;
  cudaMemcpy(&v, d, sizeof(int), cudaMemcpyDeviceToHost);
  return v;
}

int main() {
  const int n = 512;
  cudaStream_t st;
  cudaStreamCreate(&st);
  cublasHandle_t h;
  if (cublasCreate(&h) != CUBLAS_STATUS_SUCCESS) {
    std::printf("cublasCreate failed\n");
    return 2;
  }
  cublasSetStream(h, st);
  float *a0, *a, *b;
  half *h0, *ha, *hb, *cpy;
  int* info;
  cudaMalloc(&a0, sizeof(float) * n * n);
  cudaMalloc(&a, sizeof(float) * n * n);
  cudaMalloc(&b, sizeof(float) * n * n);
  cudaMalloc(&h0, sizeof(half) * n * n);
  cudaMalloc(&ha, sizeof(half) * n * n);
  cudaMalloc(&hb, sizeof(half) * n * n);
  cudaMalloc(&cpy, sizeof(half) * n * n);
  cudaMalloc(&info, sizeof(int) * 2);
  CHECK(lu_gen_matrix_c((lu_stream_t)st, n, a0, n, 7, 1, 1.5, 0, 0.0) == LU_SUCCESS);
  CHECK(lu_convert_c((lu_stream_t)st, n, n, a0, LU_F32, n, h0, LU_F16, n, 0) == LU_SUCCESS);
  cudaStreamSynchronize(st);
  const size_t fbytes = sizeof(float) * n * n, hbytes = sizeof(half) * n * n;

  // right-looking, fp32 storage, TC32 trailing updates (with the copy buffer)
  cudaMemcpy(a, a0, fbytes, cudaMemcpyDeviceToDevice);
  cudaMemcpy(b, a0, fbytes, cudaMemcpyDeviceToDevice);
  remifa::lu_nopiv_rl<float, remifa::FP32, remifa::TC32>(h, n, n, 128, a, n, info, cpy, n);
  CHECK(info_of(info) == 0);
  lu_opts o;
  lu_opts_default(&o);
  o.nb = 128;
  o.outer_update = LU_COMPUTE_TC32;
  CHECK(lu_nopiv_rl_c(&o, (lu_stream_t)st, n, n, b, LU_F32, n, info + 1, nullptr, 0, nullptr,
                      0) == LU_SUCCESS);
  cudaStreamSynchronize(st);
  CHECK(same(a, b, (size_t)n * n));
  CHECK(lu_convert_c((lu_stream_t)st, n, n, b, LU_F32, n, hb, LU_F16, n, 0) == LU_SUCCESS);
  cudaStreamSynchronize(st);
  CHECK(same(cpy, hb, (size_t)n * n));  // the fp16 copy of the factors

  // left-looking fp32 wrapper
  cudaMemcpy(a, a0, fbytes, cudaMemcpyDeviceToDevice);
  cudaMemcpy(b, a0, fbytes, cudaMemcpyDeviceToDevice);
  remifa::lu_nopiv_ll_f32(h, n, n, 64, a, n, info);
  CHECK(info_of(info) == 0);
  lu_opts_default(&o);
  o.nb = 64;
  CHECK(lu_nopiv_ll_c(&o, (lu_stream_t)st, n, n, b, LU_F32, n, info + 1, nullptr, 0, nullptr,
                      0) == LU_SUCCESS);
  cudaStreamSynchronize(st);
  CHECK(same(a, b, (size_t)n * n));

  // left-looking fp16 storage, TC32 updates; and the OP = fp32 wrapper
  for (int op32 = 0; op32 < 2; ++op32) {
    cudaMemcpy(ha, h0, hbytes, cudaMemcpyDeviceToDevice);
    cudaMemcpy(hb, h0, hbytes, cudaMemcpyDeviceToDevice);
    if (op32)
      remifa::lu_nopiv_ll_f16_tc32xtc32_fp32xfp32_fp32xfp32(h, n, n, 128, ha, n, info);
    else
      remifa::lu_nopiv_ll_f16_tc32xtc32(h, n, n, 128, ha, n, info);
    CHECK(info_of(info) == 0);
    lu_opts_default(&o);
    o.nb = 128;
    o.outer_update = LU_COMPUTE_TC32;
    o.inner_update = LU_COMPUTE_TC32;
    o.panel_fp32 = op32;
    CHECK(lu_nopiv_ll_c(&o, (lu_stream_t)st, n, n, hb, LU_F16, n, info + 1, nullptr, 0,
                        nullptr, 0) == LU_SUCCESS);
    cudaStreamSynchronize(st);
    CHECK(same(ha, hb, (size_t)n * n));
  }

  // gemmex with fp16 operands and fp32 result (TC32)
  cudaMemcpy(a, a0, fbytes, cudaMemcpyDeviceToDevice);
  cudaMemcpy(b, a0, fbytes, cudaMemcpyDeviceToDevice);
  remifa::gemmex<remifa::CublasImpl, remifa::TC, float, half, float>(
      h, n, n, 256, -1.0f, h0, n, h0 + 256, n, 1.0f, a, n);
  cudaStreamSynchronize(st);
  CHECK(lu_gemm_update_ex_c((lu_stream_t)st, LU_COMPUTE_TC32, n, n, 256, -1.0, h0, LU_F16, n,
                            h0 + 256, LU_F16, n, 1.0, b, LU_F32, n, nullptr, 0) == LU_SUCCESS);
  cudaStreamSynchronize(st);
  CHECK(same(a, b, (size_t)n * n));

  // convert<float, half>
  remifa::convert<float, half>(st, n, n, a0, n, ha, n);
  CHECK(lu_convert_c((lu_stream_t)st, n, n, a0, LU_F32, n, hb, LU_F16, n, 0) == LU_SUCCESS);
  cudaStreamSynchronize(st);
  CHECK(same(ha, hb, (size_t)n * n));

  // lu_nopiv_panel<float, 8> on the first 8 columns / rows
  cudaMemcpy(a, a0, fbytes, cudaMemcpyDeviceToDevice);
  cudaMemcpy(b, a0, fbytes, cudaMemcpyDeviceToDevice);
  float* d;
  cudaMalloc(&d, sizeof(float) * 64);
  cudaMemcpy2D(d, 8 * sizeof(float), a0, n * sizeof(float), 8 * sizeof(float), 8,
               cudaMemcpyDeviceToDevice);
  remifa::lu_nopiv_panel<float, 8>(st, n, 8, d, 8, a, n, a, n, info);
  CHECK(lu_panel_c((lu_stream_t)st, LU_F32, n, 8, d, 8, b, n, b, n, info + 1) == LU_SUCCESS);
  cudaStreamSynchronize(st);
  CHECK(same(a, b, (size_t)n * n));

  CHECK(cudaGetLastError() == cudaSuccess);
  cublasDestroy(h);
  std::printf("failures %d\n", failures);
  return failures == 0 ? 0 : 1;
}
