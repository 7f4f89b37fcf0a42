// Internal profiling hooks (see profile.cu).
#pragma once

#include "common.cuh"

namespace lub {

// Records a CUDA event pair around its lifetime on `st` when profiling is
// on (lu_profile_begin); `bytes`/`flops` are the algorithmic work.
class ProfScope {
 public:
  ProfScope(const char* name, cudaStream_t st, double bytes = 0.0,
            double flops = 0.0);
  ~ProfScope();
  ProfScope(const ProfScope&) = delete;
  ProfScope& operator=(const ProfScope&) = delete;

 private:
  cudaStream_t st_;
  int idx_;
};

}  // namespace lub
