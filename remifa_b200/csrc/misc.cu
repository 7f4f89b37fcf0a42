// Small utilities shared by the drivers: status words, error recording,
// per-device attributes.
#include "common.cuh"
#include "kernels.cuh"

#include <cstring>
#include <mutex>
#include <unordered_map>

namespace lub {
namespace {

__global__ void fill_int_kernel(int* p, int v, int64_t count) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < count) p[i] = v;
}

// LAPACK-style info: 0, or the 1-based column of the first bad pivot;
// -1 if a bounded device-side wait gave up (err non-zero).
__global__ void finalize_info_kernel(const int* first_bad, const int* err,
                                     int* info) {
  const int f = *first_bad;
  *info = (err != nullptr && *err != 0) ? -1 : (f == kNoBadPivot) ? 0 : f;
}

std::mutex g_mu;
thread_local char g_last_error[512] = {0};

}  // namespace

void record_cuda_error(cudaError_t e, const char* what, const char* file,
                       int line) {
  std::snprintf(g_last_error, sizeof(g_last_error), "%s failed: %s (%s:%d)",
                what, cudaGetErrorString(e), file, line);
  if (std::getenv("LU_B200_VERBOSE")) std::fprintf(stderr, "[lu_b200] %s\n", g_last_error);
}

void record_message(const char* msg) {
  std::snprintf(g_last_error, sizeof(g_last_error), "%s", msg);
  if (std::getenv("LU_B200_VERBOSE")) std::fprintf(stderr, "[lu_b200] %s\n", g_last_error);
}

const char* last_error_message() { return g_last_error; }

int sm_count() {
  static std::unordered_map<int, int> cache;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 148;
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = cache.find(dev);
  if (it != cache.end()) return it->second;
  int n = 148;
  cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
  cache[dev] = n;
  return n;
}

cudaError_t set_smem_limit(const void* func, size_t bytes) {
  // The attribute is per (function, device); remember the largest value set.
  static std::unordered_map<uint64_t, size_t> done;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const uint64_t key = ((uint64_t)(uintptr_t)func) ^ ((uint64_t)dev << 56);
  {
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = done.find(key);
    if (it != done.end() && it->second >= bytes) return cudaSuccess;
  }
  if (bytes <= 48 * 1024) return cudaSuccess;
  e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)bytes);
  if (e == cudaSuccess) {
    std::lock_guard<std::mutex> lk(g_mu);
    done[key] = bytes;
  }
  return e;
}

lu_status launch_fill_int(cudaStream_t st, int* p, int v, int64_t count) {
  if (count <= 0) return LU_SUCCESS;
  fill_int_kernel<<<(unsigned)ceil_div(count, 256), 256, 0, st>>>(p, v, count);
  LUB_LAUNCH_CHECK();
  return LU_SUCCESS;
}

lu_status launch_finalize_info(cudaStream_t st, const int* first_bad,
                               const int* err, int* info) {
  finalize_info_kernel<<<1, 1, 0, st>>>(first_bad, err, info);
  LUB_LAUNCH_CHECK();
  return LU_SUCCESS;
}

namespace {

// Counts the float bit patterns whose rcp_rn differs from __frcp_rn (NaN
// results compare equal when both are NaN).  Grid-stride over [lo, hi).
__global__ void rcp_check_kernel(uint64_t lo, uint64_t hi,
                                 unsigned long long* __restrict__ bad) {
  unsigned long long local = 0;
  for (uint64_t i = lo + (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < hi;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const float d = __uint_as_float((uint32_t)i);
    const float a = rcp_rn(d), b = __frcp_rn(d);
    const bool same = (__float_as_uint(a) == __float_as_uint(b)) || (isnan(a) && isnan(b));
    local += same ? 0ull : 1ull;
  }
  if (local) atomicAdd(bad, local);
}

}  // namespace

}  // namespace lub

extern "C" LU_API lu_status lu_selfcheck_rcp_c(lu_stream_t stream, unsigned long long* d_bad) {
  if (!d_bad) return LU_ERR_INVALID_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  LUB_CUDA_TRY(cudaMemsetAsync(d_bad, 0, sizeof(unsigned long long), st));
  lub::rcp_check_kernel<<<148 * 16, 256, 0, st>>>(0ull, 1ull << 32, d_bad);
  LUB_LAUNCH_CHECK();
  return LU_SUCCESS;
}

namespace lub {
namespace {
cudaMemPool_t g_pools[64] = {};
std::mutex g_pool_mu;
}  // namespace

cudaError_t pool_malloc_async(void** p, size_t bytes, cudaStream_t st) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaMallocAsync(p, bytes, st);
  cudaMemPool_t pool = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_pool_mu);
    if (!g_pools[dev]) {
      cudaMemPoolProps props;
      std::memset(&props, 0, sizeof(props));
      props.allocType = cudaMemAllocationTypePinned;
      props.location.type = cudaMemLocationTypeDevice;
      props.location.id = dev;
      cudaMemPool_t np = nullptr;
      e = cudaMemPoolCreate(&np, &props);
      if (e != cudaSuccess) return e;
      uint64_t keep = UINT64_MAX;  // freed memory stays in the pool
      e = cudaMemPoolSetAttribute(np, cudaMemPoolAttrReleaseThreshold, &keep);
      if (e != cudaSuccess) {
        cudaMemPoolDestroy(np);
        return e;
      }
      g_pools[dev] = np;
    }
    pool = g_pools[dev];
  }
  return cudaMallocFromPoolAsync(p, bytes, pool, st);
}
}  // namespace lub

extern "C" LU_API lu_status lu_trim_memory_c(void) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return LU_ERR_NO_DEVICE;
  std::lock_guard<std::mutex> lk(lub::g_pool_mu);
  if (dev >= 0 && dev < 64 && lub::g_pools[dev]) {
    if (cudaDeviceSynchronize() != cudaSuccess) return LU_ERR_CUDA;
    if (cudaMemPoolTrimTo(lub::g_pools[dev], 0) != cudaSuccess) return LU_ERR_CUDA;
  }
  return LU_SUCCESS;
}
