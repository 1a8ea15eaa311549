// Optional per-kernel timing with CUDA events on the library stream (mb_profile*).
#include <map>
#include <string>
#include <vector>

#include "internal.h"

namespace mb {
namespace {

struct Pending {
  std::string name;
  cudaEvent_t a, b;
  double bytes, flops;
};
struct Stat {
  uint64_t launches = 0;
  double ms = 0, bytes = 0, flops = 0;
};

bool g_prof = false;
std::vector<Pending> g_pending;
std::vector<cudaEvent_t> g_pool;
std::map<std::string, Stat> g_stats;

cudaEvent_t take_event() {
  if (!g_pool.empty()) {
    cudaEvent_t e = g_pool.back();
    g_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

void drain() {
  for (auto& p : g_pending) {
    float ms = 0;
    cudaEventSynchronize(p.b);
    cudaEventElapsedTime(&ms, p.a, p.b);
    Stat& s = g_stats[p.name];
    s.launches += 1;
    s.ms += ms;
    s.bytes += p.bytes;
    s.flops += p.flops;
    g_pool.push_back(p.a);
    g_pool.push_back(p.b);
  }
  g_pending.clear();
}

}  // namespace

ProfScope::ProfScope(const char* name, double bytes, cudaStream_t stream, double flops) : slot(-1), st(stream) {
  if (!g_prof) return;
  if (g_pending.size() > 200000) drain();
  Pending p{name, take_event(), take_event(), bytes, flops};
  cudaEventRecord(p.a, st);
  g_pending.push_back(p);
  slot = int(g_pending.size()) - 1;
}

ProfScope::~ProfScope() {
  if (slot >= 0 && slot < int(g_pending.size())) cudaEventRecord(g_pending[slot].b, st);
}

}  // namespace mb

using namespace mb;

extern "C" int mb_get_stream(void** stream) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (int rc = check_init()) return rc;
  if (!stream) return MB_EINVAL;
  *stream = reinterpret_cast<void*>(g_ctx.stream);
  return MB_OK;
}

extern "C" int mb_profile(int enable) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (int rc = check_init()) return rc;
  drain();
  g_stats.clear();
  g_prof = enable != 0;
  return MB_OK;
}

extern "C" int mb_profile_report(mb_kernel_stat* stats, int cap, int* count) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (int rc = check_init()) return rc;
  if (!count || (cap > 0 && !stats)) return MB_EINVAL;
  cudaStreamSynchronize(g_ctx.stream);
  drain();
  int i = 0;
  for (auto& kv : g_stats) {
    if (i < cap) {
      std::snprintf(stats[i].name, sizeof(stats[i].name), "%s", kv.first.c_str());
      stats[i].launches = kv.second.launches;
      stats[i].total_ms = kv.second.ms;
      stats[i].bytes = kv.second.bytes;
      stats[i].flops = kv.second.flops;
    }
    ++i;
  }
  *count = i;
  return MB_OK;
}

// ---------------------------------------------------------------------------------------------
// FP64 peak probe: eight independent DFMA chains per thread on every SM, long enough to time
// with events; the denominator for kernels bound by the FP64 pipe.
// ---------------------------------------------------------------------------------------------
namespace mb {
__global__ void __launch_bounds__(256) k_dfma_probe(double* sink, int iters, double a, double b) {
  double x[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) x[j] = threadIdx.x * 1e-9 + j;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int j = 0; j < 8; ++j) x[j] = fma(x[j], a, b);
  }
  double s = 0;
#pragma unroll
  for (int j = 0; j < 8; ++j) s += x[j];
  if (s == 12345.678) sink[0] = s;  // keeps the chains alive; never true for these inputs
}
}  // namespace mb

extern "C" int mb_measure_fp64_peak(double* tflops) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (int rc = check_init()) return rc;
  if (int rc = check_not_capturing("mb_measure_fp64_peak")) return rc;
  if (!tflops) return MB_EINVAL;
  const int blocks = g_ctx.sm_count * 8, threads = 256, iters = 1 << 14;
  cudaEvent_t a, b;
  MB_CHECK_CUDA(cudaEventCreate(&a));
  MB_CHECK_CUDA(cudaEventCreate(&b));
  double best = 0;
  int rc = MB_OK;
  for (int rep = 0; rep < 4 && !rc; ++rep) {
    cudaEventRecord(a, g_ctx.stream);
    k_dfma_probe<<<blocks, threads, 0, g_ctx.stream>>>(reinterpret_cast<double*>(g_ctx.results), iters, 0.999999, 1e-7);
    cudaEventRecord(b, g_ctx.stream);
    if (cudaGetLastError() != cudaSuccess || cudaEventSynchronize(b) != cudaSuccess) {
      set_error("FP64 probe failed");
      rc = MB_EDEVICE;
      break;
    }
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    if (rep > 0) best = std::max(best, 2.0 * 8.0 * double(iters) * blocks * threads / (ms * 1e-3) / 1e12);
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  *tflops = best;
  return rc;
}
