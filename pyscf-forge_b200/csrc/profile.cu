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
  // launches recorded into a CUDA graph are not timed
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return;
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

// Register-only FP64 throughput loops (DMMA m8n8k4 and DFMA), used to
// measure the FP64 roofline denominator on the running GPU.
__global__ void k_peak_dmma(double* sink, int iters) {
  double c[8][2];
  for (int t = 0; t < 8; ++t) c[t][0] = c[t][1] = 0.0;
  const double a = 1e-3 * threadIdx.x, b = 1e-3 * blockIdx.x;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int t = 0; t < 8; ++t)
      asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                   : "+d"(c[t][0]), "+d"(c[t][1])
                   : "d"(a), "d"(b));
  }
  double s = 0.0;
  for (int t = 0; t < 8; ++t) s += c[t][0] + c[t][1];
  if (s == 1234.5678) sink[0] = s;
}

__global__ void k_peak_dfma(double* sink, int iters) {
  double c[8];
  for (int t = 0; t < 8; ++t) c[t] = threadIdx.x * 1e-3 + t;
  const double a = 1.0000001, b = 1e-9;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int t = 0; t < 8; ++t) c[t] = fma(c[t], a, b);
  }
  double s = 0.0;
  for (int t = 0; t < 8; ++t) s += c[t];
  if (s == 1234.5678) sink[0] = s;
}

static __device__ double g_peak_sink[1];

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

int csffci_fp64_peak(int kind, int iters, double* tflops, cudaStream_t stream) {
  CSF_REQUIRE(tflops != nullptr && iters > 0 && kind >= 0 && kind <= 2, "fp64_peak: bad arguments");
  int dev = 0, nsm = 148;
  CSF_CUDA(cudaGetDevice(&dev));
  CSF_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  double* sink = nullptr;
  CSF_CUDA(cudaGetSymbolAddress((void**)&sink, g_peak_sink));
  cudaEvent_t a, b;
  CSF_CUDA(cudaEventCreate(&a));
  CSF_CUDA(cudaEventCreate(&b));
  // kind 2: one CTA of 17 warps per SM (a scheduler with 5 warps)
  const int blocks = kind == 2 ? nsm : nsm * 2, threads = kind == 2 ? 544 : 256;
  if (kind != 1) k_peak_dmma<<<blocks, threads, 0, stream>>>(sink, 64);
  else k_peak_dfma<<<blocks, threads, 0, stream>>>(sink, 64);
  cudaEventRecord(a, stream);
  if (kind != 1) k_peak_dmma<<<blocks, threads, 0, stream>>>(sink, iters);
  else k_peak_dfma<<<blocks, threads, 0, stream>>>(sink, iters);
  cudaEventRecord(b, stream);
  CSF_CUDA(cudaEventSynchronize(b));
  float ms = 0.f;
  CSF_CUDA(cudaEventElapsedTime(&ms, a, b));
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  const double warps = (double)blocks * threads / 32.0;
  const double flops = kind != 1 ? 2.0 * 8 * 8 * 4 * 8 * (double)iters * warps
                                 : 2.0 * 8 * (double)iters * blocks * threads;
  *tflops = flops / (ms * 1e-3) / 1e12;
  return check_launch("fp64_peak");
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
