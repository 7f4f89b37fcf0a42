// FP64 iterative refinement that allocates no memory (new; no counterpart in
// the reference, whose drivers cudaMalloc and cudaFree on every call,
// src/lu_nopiv.hxx:111,205).
//
// lu_refine_c needs a few hundred KB of device scratch per call (residual
// and correction vectors, column-chunk partial sums, three max accumulators)
// and takes it from the caller or from cudaMallocAsync.  Some callers can do
// neither: a service whose caching allocator has already reserved the GPU's
// memory for itself, code that runs where a device allocation would stall
// or fail (a fixed-footprint real-time loop, a library callback that must
// not touch the allocator), or a host language binding with no way to hand
// over device memory.  lu_refine_static_c serves them from one scratch array
// compiled into this library, g_refine_scratch, sized for n <= 4096.
//
// Rules of use:
//   * The first call on each device (with that device current) looks up the
//     array's device address with cudaGetSymbolAddress.  That lookup may load
//     this module onto the device, so make the first call before any stream
//     capture begins.
//   * The array is shared by every call on a device: two calls in flight at
//     once on one device (different streams or host threads) race on it and
//     give wrong results.  Serialise them.
//   * No part of the array must start at zero: the max accumulators are
//     cleared on the stream before each use and every vector and partial
//     sum is written before it is read.
//   * n > LU_REFINE_STATIC_MAX_N is rejected with LU_ERR_INVALID_ARG (the
//     message is in lu_last_error); nothing is enqueued.
#include "common.cuh"
#include "lu_b200.h"

#include <mutex>

using namespace lub;

namespace {

constexpr size_t kScratchBytes = LU_REFINE_STATIC_SCRATCH_BYTES;
constexpr int kMaxDevices = 64;

__device__ __align__(256) unsigned char g_refine_scratch[kScratchBytes];

std::mutex g_mu;
void* g_scratch_ptr[kMaxDevices] = {};

// Device address of g_refine_scratch on the current device (looked up once).
lu_status scratch_for_current_device(void** out) {
  int dev = 0;
  LUB_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return LU_ERR_NO_DEVICE;
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    LUB_CUDA_TRY(cudaGetSymbolAddress(&p, g_refine_scratch));
    g_scratch_ptr[dev] = p;
  }
  *out = g_scratch_ptr[dev];
  return LU_SUCCESS;
}

}  // namespace

extern "C" {

LU_API lu_status lu_refine_static_c(lu_stream_t stream, int64_t n, const float* d_a,
                                    int64_t lda, const float* d_lu, int64_t ldlu,
                                    const double* d_b, double* d_x, double tol,
                                    int max_iter, int* iters, double* berr) {
  if (n > LU_REFINE_STATIC_MAX_N) {
    record_message("lu_refine_static_c: n exceeds LU_REFINE_STATIC_MAX_N (4096); "
                   "use lu_refine_c with a workspace");
    return LU_ERR_INVALID_ARG;
  }
  size_t need = 0;
  LUB_TRY(lu_refine_workspace_size(n < 0 ? 0 : n, &need));
  if (need > kScratchBytes) return LU_ERR_WORKSPACE;
  if (n <= 0) {
    // argument checks and the n == 0 early return of the workspace path
    return lu_refine_c(stream, n, d_a, lda, d_lu, ldlu, d_b, d_x, tol, max_iter,
                       iters, berr, nullptr, 0);
  }
  void* scratch = nullptr;
  LUB_TRY(scratch_for_current_device(&scratch));
  return lu_refine_c(stream, n, d_a, lda, d_lu, ldlu, d_b, d_x, tol, max_iter,
                     iters, berr, scratch, kScratchBytes);
}

}  // extern "C"
