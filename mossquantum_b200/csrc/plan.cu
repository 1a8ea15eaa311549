// Prepared execution: device-side parameters and results, CUDA-graph capture and replay
// on the library stream, and the autotuner for the fused passes' tile/register widths.
//
// The reference prepares plans and sweeps on the host (src/execution/execution_plans.jl,
// experiments.jl). Here a caller runs a sequence once eagerly (building schedules,
// specialised kernels and reduction plans), records the same sequence into a CUDA graph and
// replays it with new parameters: one graph launch per evaluation of a whole batch.
#include <array>
#include <cstring>
#include <vector>

#include "internal.h"

struct mb_graph_s {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

using namespace mb;

extern "C" int mb_theta_upload(mb_circuit c, const double* theta, size_t ntheta, int rows) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (int rc = check_init()) return rc;
  if (int rc = check_not_capturing("mb_theta_upload")) return rc;
  if (!c || (!theta && ntheta) || rows < 1) return MB_EINVAL;
  return theta_stage(c, theta, ntheta, rows);
}

extern "C" int mb_buffer_alloc(size_t bytes, void** dev) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (int rc = check_init()) return rc;
  if (int rc = check_not_capturing("mb_buffer_alloc")) return rc;
  if (!dev) return MB_EINVAL;
  int rc = dev_alloc(dev, bytes);
  if (rc) return rc;
  MB_CHECK_CUDA(cudaMemsetAsync(*dev, 0, bytes, g_ctx.stream));
  MB_CHECK_CUDA(cudaStreamSynchronize(g_ctx.stream));
  return MB_OK;
}

extern "C" int mb_buffer_free(void* dev) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (!g_ctx.init || !dev) return MB_OK;
  dev_free(dev);
  return MB_OK;
}

extern "C" int mb_buffer_download(const void* dev, void* host, size_t bytes) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (int rc = check_init()) return rc;
  if (int rc = check_not_capturing("mb_buffer_download")) return rc;
  if ((!dev || !host) && bytes) return MB_EINVAL;
  MB_CHECK_CUDA(cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, g_ctx.stream));
  MB_CHECK_CUDA(cudaStreamSynchronize(g_ctx.stream));
  return MB_OK;
}

extern "C" int mb_expect_to_device(mb_observable o, mb_state s, double* dev_out) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (int rc = check_init()) return rc;
  if (!o || !s || !dev_out) return MB_EINVAL;
  if (int rc = validate_observable(o, s)) return rc;
  if (s->batch == 0) return MB_OK;
  const int is_dm = s->kind == MB_DENSITY || s->kind == MB_BATCH_DENSITY;
  double2* out = reinterpret_cast<double2*>(dev_out);
  return (!is_dm && o->pauli_ok) ? expect_pauli(o, s, out) : expect_keys(o, s, out);
}

extern "C" int mb_graph_begin(void) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (int rc = check_init()) return rc;
  if (g_ctx.capturing) {
    set_error("a graph recording is already in progress");
    return MB_EINVAL;
  }
  MB_CHECK_CUDA(cudaStreamSynchronize(g_ctx.stream));
  MB_CHECK_CUDA(cudaStreamBeginCapture(g_ctx.stream, cudaStreamCaptureModeThreadLocal));
  g_ctx.capturing = true;
  return MB_OK;
}

extern "C" int mb_graph_end(mb_graph* out) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (int rc = check_init()) return rc;
  if (!g_ctx.capturing || !out) {
    set_error("no graph recording in progress");
    return MB_EINVAL;
  }
  g_ctx.capturing = false;
  auto g = new mb_graph_s();
  cudaError_t e = cudaStreamEndCapture(g_ctx.stream, &g->graph);
  if (e == cudaSuccess) e = cudaGraphInstantiate(&g->exec, g->graph, 0);
  if (e != cudaSuccess) {
    cudaGetLastError();
    if (g->graph) cudaGraphDestroy(g->graph);
    delete g;
    set_error("graph recording failed: %s", cudaGetErrorString(e));
    return MB_EDEVICE;
  }
  *out = g;
  return MB_OK;
}

extern "C" int mb_graph_launch(mb_graph g) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (int rc = check_init()) return rc;
  if (!g) return MB_EINVAL;
  MB_CHECK_CUDA(cudaGraphLaunch(g->exec, g_ctx.stream));
  ++launch_counter();
  return MB_OK;
}

extern "C" int mb_graph_free(mb_graph g) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (!g) return MB_OK;
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->graph) cudaGraphDestroy(g->graph);
  delete g;
  return MB_OK;
}

// Candidate widths: tile bits t (shared-memory tile of 2^t amplitudes) and register bits R
// (amplitudes per thread 2^R, i.e. how many gate qubits one register stage fuses).
extern "C" int mb_autotune(mb_circuit c, mb_state s, const double* theta, size_t ntheta, int flags, int* best_t,
                           int* best_r, double* best_ms) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (int rc = check_init()) return rc;
  if (int rc = check_not_capturing("mb_autotune")) return rc;
  if (!c || !s || !best_t || !best_r || !best_ms) return MB_EINVAL;
  const int dm = s->kind == MB_DENSITY || s->kind == MB_BATCH_DENSITY;
  const int N = dm ? 2 * s->n : s->n;
  int t0 = 0, r0 = 0, f0 = 1;
  mb_tuning_get(N, &t0, &r0);
  mb_tuning_get_fusion(N, &f0);
  std::vector<std::array<int, 3>> cand;
  const bool jit = jit_sizes(N);
  if (jit) {
    // specialised kernels: tiles of 2^10 and 2^11 amplitudes with bind-time fusion, then the
    // better of the two without fusion (each candidate compiles its own kernels)
    cand.push_back({10, 3, 1});
    cand.push_back({11, 3, 1});
    if (!((t0 == 10 || t0 == 11) && r0 == 3)) cand.push_back({t0, r0, 1});
  } else {
    for (int f : {1, 0})
      for (auto tr : {std::array<int, 2>{12, 4}, {11, 4}, {10, 4}, {12, 3}, {11, 3}, {10, 3}}) cand.push_back({tr[0], tr[1], f});
  }
  double best = 1e300;
  int bt = t0, br = r0, bf = f0;
  cudaEvent_t a, b;
  MB_CHECK_CUDA(cudaEventCreate(&a));
  MB_CHECK_CUDA(cudaEventCreate(&b));
  int rc = MB_OK;
  // times one candidate (a warm-up apply builds its schedule and kernels, then two timed
  // applies); false on an error that ends the search
  auto run = [&](const std::array<int, 3>& cd) -> bool {
    if (cd[0] > N) return true;
    if ((rc = mb_tuning_set(N, cd[0], cd[1]))) return false;
    if ((rc = mb_tuning_set_fusion(N, cd[2]))) return false;
    if ((rc = mb_apply(c, s, theta, ntheta, flags & ~MB_APPLY_PLAIN))) {
      rc = MB_OK;  // a width this circuit cannot use (e.g. no specialised kernels): skip it
      return true;
    }
    int et = 0, er = 0;
    mb_tuning_get(N, &et, &er);
    if (et != cd[0] || er != cd[1]) return true;  // the library fell back to another width
    cudaEventRecord(a, g_ctx.stream);
    for (int k = 0; k < 2 && !rc; ++k) rc = mb_apply(c, s, theta, ntheta, flags & ~MB_APPLY_PLAIN);
    cudaEventRecord(b, g_ctx.stream);
    cudaEventSynchronize(b);
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    if (!rc && ms / 2 < best) {
      best = ms / 2;
      bt = cd[0];
      br = cd[1];
      bf = cd[2];
    }
    return rc == MB_OK;
  };
  bool ok = true;
  for (const auto& cd : cand)
    if (!(ok = run(cd))) break;
  // specialised sizes: the better fused shape once more without fusion
  if (ok && jit && best < 1e300) run({bt, br, 0});
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  mb_tuning_set(N, bt, br);
  mb_tuning_set_fusion(N, bf);
  *best_t = bt;
  *best_r = br;
  *best_ms = best;
  return rc;
}
