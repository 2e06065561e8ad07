// RAII event pair around a kernel launch when profiling is enabled.
#pragma once
#include <cuda_runtime.h>

namespace csffci {
bool prof_on();
struct ProfScope {
  ProfScope(const char* name, cudaStream_t s);
  ~ProfScope();
  const char* name_;
  cudaStream_t stream_;
  cudaEvent_t a_, b_;
};
}  // namespace csffci
