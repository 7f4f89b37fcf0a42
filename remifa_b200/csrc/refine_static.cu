// FP64 iterative refinement that allocates no memory (new; no counterpart in
// the reference, whose drivers cudaMalloc and cudaFree on every call,
// src/lu_nopiv.hxx:111,205).
//
// lu_refine_c needs a few hundred KB of device scratch per call (residual
// and correction vectors, column-chunk partial sums, three max accumulators)
// and takes it from the caller or from a stream-ordered memory pool.  Some callers can do
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
//     capture begins.  Every call also synchronises its stream (it reads the
//     backward error back once per iteration), so no call can be made while
//     the stream is being captured.
//   * The address is kept per device together with the identity of the CUDA
//     context it was looked up in (cuCtxGetId); after cudaDeviceReset the
//     context is a new one and the next call looks the address up again.
//   * The array is shared by every call on a device: two calls in flight at
//     once on one device (different streams or host threads) race on it and
//     give wrong results.  Serialise them.
//   * No part of the array must start at zero: the max accumulators are
//     cleared on the stream before each use and every vector and partial
//     sum is written before it is read.
//   * n > LU_REFINE_STATIC_MAX_N is rejected with LU_ERR_INVALID_ARG (the
//     message is in lu_last_error); nothing is enqueued.  Bad arguments are
//     rejected before any device call, as lu_refine_c rejects them.
#include "common.cuh"
#include "solve.cuh"
#include "lu_b200.h"

#include <cuda.h>
#include <algorithm>
#include <mutex>

using namespace lub;

namespace {

constexpr size_t kScratchBytes = LU_REFINE_STATIC_SCRATCH_BYTES;
constexpr int kMaxDevices = 64;

__device__ __align__(256) unsigned char g_refine_scratch[kScratchBytes];

struct ScratchEntry {
  unsigned long long ctx_id;  // identity of the context the lookup ran in
  void* ptr;                  // device address of g_refine_scratch there
};

std::mutex g_mu;
ScratchEntry g_scratch[kMaxDevices] = {};

using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

// Identity of the calling thread's current context (0 if there is none
// yet), through driver entry points fetched by the runtime (this library
// does not link libcuda).
lu_status current_context_id(unsigned long long* id) {
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) ==
            cudaSuccess && q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<CtxGetCurrentFn>(p);
    if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<CtxGetIdFn>(p);
  });
  if (!get_current || !get_id) {
    record_message("lu_refine_static_c: cuCtxGetCurrent / cuCtxGetId unavailable");
    return LU_ERR_CUDA;
  }
  CUcontext ctx = nullptr;
  if (get_current(&ctx) != CUDA_SUCCESS) return LU_ERR_CUDA;
  *id = 0;
  if (ctx && get_id(ctx, id) != CUDA_SUCCESS) return LU_ERR_CUDA;
  return LU_SUCCESS;
}

// Device address of g_refine_scratch on the current device: looked up once
// per device and context (the set-up), reused while that context lives.
lu_status scratch_for_current_device(void** out) {
  int dev = 0;
  LUB_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return LU_ERR_NO_DEVICE;
  std::lock_guard<std::mutex> lk(g_mu);
  unsigned long long id = 0;
  LUB_TRY(current_context_id(&id));
  ScratchEntry& e = g_scratch[dev];
  if (id == 0 || e.ptr == nullptr || e.ctx_id != id) {
    void* p = nullptr;
    LUB_CUDA_TRY(cudaGetSymbolAddress(&p, g_refine_scratch));
    LUB_TRY(current_context_id(&id));  // the lookup made the context current
    e.ctx_id = id;
    e.ptr = p;
  }
  *out = e.ptr;
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
  const int64_t one = std::max<int64_t>(1, n);
  LUB_TRY(refine_check_args(n, 1, d_a, lda, d_lu, ldlu, d_b, one, d_x, one, 0, tol,
                            max_iter));
  size_t need = 0;
  LUB_TRY(lu_refine_workspace_size(n, &need));
  if (need > kScratchBytes) {
    record_message("lu_refine_static_c: the refinement layout for this n exceeds "
                   "LU_REFINE_STATIC_SCRATCH_BYTES");
    return LU_ERR_WORKSPACE;
  }
  if (n == 0) {
    if (iters) *iters = 0;
    if (berr) *berr = 0.0;
    return LU_SUCCESS;
  }
  LUB_TRY(refine_check_device());
  void* scratch = nullptr;
  LUB_TRY(scratch_for_current_device(&scratch));
  return lu_refine_c(stream, n, d_a, lda, d_lu, ldlu, d_b, d_x, tol, max_iter,
                     iters, berr, scratch, kScratchBytes);
}

}  // extern "C"
