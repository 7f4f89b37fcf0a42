// Self-tests of the bounded device waits (no counterpart in the reference).
//
// Every wait in this library's kernels that depends on another role or
// another CTA is bounded, so that a lost producer ends in an error status
// the host reads instead of a hung GPU:
//   * the tensor-core update's mbarrier waits (sm100::mbar_wait): on expiry
//     the kernel records an error code, each role unwinds -- waiting, with
//     the same bound, for the copies and MMAs it issued itself -- the TMEM
//     is freed, and a factorization reports info = -1 (LU_ERR_TIMEOUT);
//   * the triangular solve's waits for earlier row blocks: on expiry the
//     entries still pending become NaN and every other wait of the solve
//     gives up at once, so the solve ends with NaN in its result.
// These entry points make those waits run out on purpose and by
// construction: the update runs with its TMA producer withheld (it issues
// no loads, so the barriers the consumers wait on never complete), the
// solve with the row block solved first withholding its solution; each
// with a short bound.  Nothing faults: no copy is in flight when a CTA
// ends, no MMA when its TMEM is freed.
#include "common.cuh"
#include "kernels.cuh"
#include "solve.cuh"
#include "tc_gemm.cuh"
#include "lu_b200.h"

using namespace lub;

namespace {

constexpr int64_t kM = 512, kN = 512, kK = 64;  // 4 x 2 tiles of 128 x 256

lu_status check_device_here() {
  int dev = 0, major = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return LU_ERR_NO_DEVICE;
  if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev) != cudaSuccess)
    return LU_ERR_NO_DEVICE;
  return major == 10 ? LU_SUCCESS : LU_ERR_NO_DEVICE;
}

}  // namespace

extern "C" {

LU_API lu_status lu_selftest_wait_update_c(lu_stream_t stream, long long wait_cycles,
                                           int streaming, void* d_scratch, size_t bytes,
                                           int* d_out) {
  if (wait_cycles <= 0 || !d_scratch || !d_out ||
      bytes < (size_t)LU_SELFTEST_SCRATCH_BYTES || (uintptr_t)d_scratch % 1024 != 0)
    return LU_ERR_INVALID_ARG;
  LUB_TRY(check_device_here());
  cudaStream_t st = (cudaStream_t)stream;
  char* ws = static_cast<char*>(d_scratch);
  int* err = reinterpret_cast<int*>(ws);
  int* first_bad = err + 1;
  char* A = ws + 1024;                         // kM x kK fp16, row-major
  char* B = A + kM * kK * 2;                   // kN x kK fp16, column-major
  float* C = reinterpret_cast<float*>(B + kN * kK * 2);  // kM x kN fp32
  LUB_TRY(launch_fill_int(st, err, 0, 1));
  LUB_TRY(launch_fill_int(st, first_bad, kNoBadPivot, 1));
  LUB_CUDA_TRY(cudaMemsetAsync(A, 0, (size_t)(kM + kN) * kK * 2 + kM * kN * 4, st));
  LUB_TRY(launch_tc_update_withheld(st, kM, kN, kK, A, kK, B, kK, C, kM, err, wait_cycles,
                                    streaming ? 4 : 1));
  LUB_CUDA_TRY(cudaMemcpyAsync(d_out, err, sizeof(int), cudaMemcpyDeviceToDevice, st));
  return launch_finalize_info(st, first_bad, err, d_out + 1);
}

LU_API lu_status lu_selftest_wait_solve_c(lu_stream_t stream, unsigned long long wait_ns,
                                          int64_t n, const float* d_lu, int64_t ldlu,
                                          double* d_x, void* d_scratch, size_t bytes,
                                          unsigned* d_expired) {
  if (wait_ns == 0 || n < 128 || ldlu < n || !d_lu || !d_x || !d_scratch || !d_expired)
    return LU_ERR_INVALID_ARG;
  if (bytes < trsm_ws_bytes(n, 1)) return LU_ERR_WORKSPACE;
  LUB_TRY(check_device_here());
  cudaStream_t st = (cudaStream_t)stream;
  unsigned* sync = static_cast<unsigned*>(d_scratch);
  double* B = reinterpret_cast<double*>(static_cast<char*>(d_scratch) + trsm_sync_bytes(1));
  // the unit-lower solve L x = b with the first row block withheld
  LUB_TRY(launch_trsm(st, n, d_lu, ldlu, d_x, n, 1, false, false, sync, B, wait_ns, 0));
  LUB_CUDA_TRY(cudaMemcpyAsync(d_expired, sync + 1, sizeof(unsigned),
                               cudaMemcpyDeviceToDevice, st));
  return LU_SUCCESS;
}

}  // extern "C"
