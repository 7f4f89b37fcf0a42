// Lightweight in-library profiling: CUDA events recorded on the launching
// stream around each kernel class, plus a count of every kernel this library
// launches.  Off by default; lu_profile_begin() turns it on.  The reference
// has only wall-clock timing around the whole factorization
// (tests/testing_lu_gpu.hxx:1106-1260).
#include "common.cuh"
#include "profile.cuh"

#include <atomic>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

namespace lub {
namespace {

struct Rec {
  const char* name;
  cudaEvent_t a, b;
  double bytes, flops;
  cudaStream_t st;
};

std::atomic<long long> g_launches{0};
std::atomic<bool> g_on{false};
std::mutex g_mu;
std::vector<Rec> g_recs;
std::vector<cudaEvent_t> g_pool;

cudaEvent_t get_event() {
  if (!g_pool.empty()) {
    cudaEvent_t e = g_pool.back();
    g_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

}  // namespace

void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

ProfScope::ProfScope(const char* name, cudaStream_t st, double bytes,
                     double flops)
    : st_(st), idx_(-1) {
  if (!g_on.load(std::memory_order_relaxed)) return;
  std::lock_guard<std::mutex> lk(g_mu);
  Rec r{name, get_event(), get_event(), bytes, flops, st};
  cudaEventRecord(r.a, st);
  g_recs.push_back(r);
  idx_ = (int)g_recs.size() - 1;
}

ProfScope::~ProfScope() {
  if (idx_ < 0) return;
  std::lock_guard<std::mutex> lk(g_mu);
  if (idx_ < (int)g_recs.size()) cudaEventRecord(g_recs[idx_].b, st_);
}

}  // namespace lub

using namespace lub;

extern "C" {

LU_API void lu_profile_begin(void) {
  std::lock_guard<std::mutex> lk(g_mu);
  for (auto& r : g_recs) {
    g_pool.push_back(r.a);
    g_pool.push_back(r.b);
  }
  g_recs.clear();
  g_on.store(true);
}

LU_API int lu_profile_end(lu_profile_entry* out, int max_entries) {
  g_on.store(false);
  std::lock_guard<std::mutex> lk(g_mu);
  std::map<std::string, lu_profile_entry> agg;
  for (auto& r : g_recs) {
    cudaEventSynchronize(r.b);
    float ms = 0.0f;
    if (cudaEventElapsedTime(&ms, r.a, r.b) != cudaSuccess) ms = 0.0f;
    auto& e = agg[r.name];
    std::strncpy(e.name, r.name, sizeof(e.name) - 1);
    e.launches += 1;
    e.total_ms += ms;
    e.bytes += r.bytes;
    e.flops += r.flops;
  }
  int k = 0;
  for (auto& kv : agg) {
    if (out && k < max_entries) out[k] = kv.second;
    ++k;
  }
  return k;
}

LU_API int lu_profile_trace(lu_trace_entry* out, int max_entries) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (g_recs.empty()) return 0;
  std::map<cudaStream_t, int> ids;
  int k = 0;
  for (auto& r : g_recs) {
    if (g_on.load()) break;  // only after lu_profile_end
    if (out && k < max_entries) {
      lu_trace_entry& e = out[k];
      std::memset(&e, 0, sizeof(e));
      std::strncpy(e.name, r.name, sizeof(e.name) - 1);
      auto it = ids.find(r.st);
      if (it == ids.end()) it = ids.emplace(r.st, (int)ids.size()).first;
      e.stream = it->second;
      float t0 = 0.0f, t1 = 0.0f;
      cudaEventSynchronize(r.b);
      if (cudaEventElapsedTime(&t0, g_recs[0].a, r.a) != cudaSuccess) t0 = 0.0f;
      if (cudaEventElapsedTime(&t1, g_recs[0].a, r.b) != cudaSuccess) t1 = 0.0f;
      e.start_ms = t0;
      e.end_ms = t1;
    }
    ++k;
  }
  return k;
}

LU_API long long lu_launch_count(void) {
  return g_launches.load(std::memory_order_relaxed);
}

}  // extern "C"
