// Per-kernel CUDA-event timing (tracing hook).  When enabled on the
// calling host thread, the main kernels record an event pair around their
// launch on the launching stream; csffci_profile_report() synchronises and
// returns "name count total_ms" lines.  Disabled by default: zero cost.
#include <map>
#include <string>
#include <vector>

#include "common.cuh"
#include "profile.cuh"

namespace csffci {

struct ProfState {
  bool on = false;
  std::map<std::string, std::vector<std::pair<cudaEvent_t, cudaEvent_t>>> ev;
};

static thread_local ProfState g_prof;

bool prof_on() { return g_prof.on; }

void prof_record(const char* name, cudaEvent_t a, cudaEvent_t b) { g_prof.ev[name].push_back({a, b}); }

ProfScope::ProfScope(const char* name, cudaStream_t s) : name_(name), stream_(s), a_(nullptr), b_(nullptr) {
  if (!g_prof.on) return;
  if (cudaEventCreate(&a_) != cudaSuccess || cudaEventCreate(&b_) != cudaSuccess) {
    a_ = b_ = nullptr;
    return;
  }
  cudaEventRecord(a_, stream_);
}

ProfScope::~ProfScope() {
  if (!a_) return;
  cudaEventRecord(b_, stream_);
  prof_record(name_, a_, b_);
}

}  // namespace csffci

using namespace csffci;

extern "C" {

int csffci_profile_enable(int on) {
  for (auto& kv : g_prof.ev)
    for (auto& p : kv.second) {
      cudaEventDestroy(p.first);
      cudaEventDestroy(p.second);
    }
  g_prof.ev.clear();
  g_prof.on = on != 0;
  return CSFFCI_OK;
}

int csffci_profile_report(char* buf, size_t len) {
  std::string out;
  for (auto& kv : g_prof.ev) {
    double tot = 0.0;
    for (auto& p : kv.second) {
      CSF_CUDA(cudaEventSynchronize(p.second));
      float ms = 0.f;
      CSF_CUDA(cudaEventElapsedTime(&ms, p.first, p.second));
      tot += ms;
    }
    char line[256];
    snprintf(line, sizeof(line), "%s %zu %.6f\n", kv.first.c_str(), kv.second.size(), tot);
    out += line;
  }
  if (buf && len) {
    snprintf(buf, len, "%s", out.c_str());
  }
  return CSFFCI_OK;
}

}  // extern "C"
