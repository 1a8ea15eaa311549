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
  double bytes;
};
struct Stat {
  uint64_t launches = 0;
  double ms = 0, bytes = 0;
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
    g_pool.push_back(p.a);
    g_pool.push_back(p.b);
  }
  g_pending.clear();
}

}  // namespace

ProfScope::ProfScope(const char* name, double bytes, cudaStream_t stream) : slot(-1), st(stream) {
  if (!g_prof) return;
  if (g_pending.size() > 200000) drain();
  Pending p{name, take_event(), take_event(), bytes};
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
    }
    ++i;
  }
  *count = i;
  return MB_OK;
}
