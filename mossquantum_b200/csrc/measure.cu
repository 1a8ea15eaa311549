// Mid-circuit measurement and post-selection on the device (src/execution/measurement.jl:4-201,
// src/execution/post_selection.jl:3-112).
//
// The outcome probabilities of one qubit come from the marginal kernel (one read of the
// state); the host draws the outcome with its own random stream, exactly like the
// reference's discrete_sample over device-computed probabilities; the collapse is one
// per-sample 2x2 operator (the projector, or |0><i| with automatic reset, divided by
// sqrt(p)) applied by the plain gate kernel, on the row and column bits of a density matrix.
// Removing the measured qubit writes the outcome's slice into a state one qubit smaller.
#include <cmath>
#include <vector>

#include "internal.h"

namespace mb {
namespace {

__global__ void k_remove_qubit(const double2* __restrict__ src, double2* __restrict__ dst, int n, int q,
                               const int* __restrict__ outcomes, const double* __restrict__ scales, int nsamples) {
  const int64_t half = int64_t(1) << (n - 1);
  const int64_t total = half * nsamples;
  for (int64_t g = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; g < total; g += int64_t(gridDim.x) * blockDim.x) {
    const int b = int(g / half);
    const int64_t j = g - int64_t(b) * half;
    const int64_t low = j & ((int64_t(1) << q) - 1);
    const int64_t i = ((j >> q) << (q + 1)) | (int64_t(outcomes[b]) << q) | low;
    const double2 x = src[(int64_t(b) << n) + i];
    dst[int64_t(b) * half + j] = make_double2(x.x * scales[b], x.y * scales[b]);
  }
}

__global__ void k_scale_samples(double2* __restrict__ v, int64_t elems, int nsamples, const double* __restrict__ sc) {
  const int64_t total = elems * nsamples;
  for (int64_t g = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; g < total; g += int64_t(gridDim.x) * blockDim.x) {
    const double s = sc[g / elems];
    const double2 x = v[g];
    v[g] = make_double2(x.x * s, x.y * s);
  }
}

int check_qubit(mb_state s, int qubit) {
  if (!s) return MB_EINVAL;
  if (qubit < 0 || qubit >= s->n) {
    set_error("qubit position must be between 1 and %d", s->n);
    return MB_EINVAL;
  }
  return MB_OK;
}

}  // namespace
}  // namespace mb

using namespace mb;

extern "C" int mb_qubit_weights(mb_state s, int qubit, double* w) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (int rc = check_init()) return rc;
  if (int rc = check_not_capturing("mb_qubit_weights")) return rc;
  if (int rc = check_qubit(s, qubit)) return rc;
  if (!w) return MB_EINVAL;
  if (s->batch == 0) return MB_OK;
  const int is_dm = s->kind == MB_DENSITY || s->kind == MB_BATCH_DENSITY;
  const size_t bytes = sizeof(double) * 2 * size_t(s->batch);
  double* d = nullptr;
  int rc = dev_alloc((void**)&d, bytes);
  if (rc) return rc;
  cudaStream_t st = g_ctx.stream;
  cudaMemsetAsync(d, 0, bytes, st);
  cudaMemsetAsync(g_ctx.flags, 0, sizeof(unsigned) * 2, st);
  rc = launch_marginal(s->d, s->n, is_dm, s->batch, &qubit, 1, d, g_ctx.flags, std::sqrt(2.220446049250313e-16), st);
  if (!rc) {
    cudaMemcpyAsync(w, d, bytes, cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) {
      set_error("qubit weights: %s", cudaGetErrorString(cudaGetLastError()));
      rc = MB_EDEVICE;
    }
  }
  dev_free(d);
  return rc;
}

extern "C" int mb_collapse(mb_state s, int qubit, const int* outcomes, const double* probs, int auto_reset) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (int rc = check_init()) return rc;
  if (int rc = check_not_capturing("mb_collapse")) return rc;
  if (int rc = check_qubit(s, qubit)) return rc;
  if (s->batch == 0) return MB_OK;
  if (!outcomes || !probs) return MB_EINVAL;
  const int B = s->batch;
  // Validate every sample before touching the state.
  std::vector<double2> m(size_t(B) * 4, make_double2(0.0, 0.0));
  for (int b = 0; b < B; ++b) {
    if ((outcomes[b] != 0 && outcomes[b] != 1) || !(probs[b] > 0) || !std::isfinite(probs[b])) {
      set_error("sample %d: outcome must be 0 or 1 with a positive finite probability", b);
      return MB_EINVAL;
    }
    const double sc = 1.0 / std::sqrt(probs[b]);
    const int i = outcomes[b];
    // column-major 2x2: |0><i| (automatic reset) or |i><i|, scaled
    if (auto_reset) m[size_t(b) * 4 + 0 + 2 * i] = make_double2(sc, 0.0);
    else m[size_t(b) * 4 + i + 2 * i] = make_double2(sc, 0.0);
  }
  double2* d = nullptr;
  int rc = dev_alloc((void**)&d, sizeof(double2) * m.size());
  if (rc) return rc;
  cudaStream_t st = g_ctx.stream;
  cudaMemcpyAsync(d, m.data(), sizeof(double2) * m.size(), cudaMemcpyHostToDevice, st);
  const int is_dm = s->kind == MB_DENSITY || s->kind == MB_BATCH_DENSITY;
  Pos p{};
  p.k = 1;
  p.p[0] = qubit;
  rc = launch_dense(s->d, s->elems, B, p, d, 4, MAT_PLAIN, st);
  if (!rc && is_dm) {
    p.p[0] = qubit + s->n;
    rc = launch_dense(s->d, s->elems, B, p, d, 4, MAT_CONJ, st);
  }
  if (!rc && cudaStreamSynchronize(st) != cudaSuccess) {
    set_error("collapse: %s", cudaGetErrorString(cudaGetLastError()));
    rc = MB_EDEVICE;
  }
  dev_free(d);
  return rc;
}

extern "C" int mb_remove_qubit(mb_state src, int qubit, const int* outcomes, const double* scales, mb_state dst) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (int rc = check_init()) return rc;
  if (int rc = check_not_capturing("mb_remove_qubit")) return rc;
  if (int rc = check_qubit(src, qubit)) return rc;
  if (!dst || src == dst) return MB_EINVAL;
  const bool pure = src->kind == MB_PURE || src->kind == MB_BATCH_PURE;
  if (!pure || dst->kind != src->kind || dst->n != src->n - 1 || dst->batch != src->batch) {
    set_error("removing a qubit needs a pure source and a pure destination of n-1 qubits and the same batch");
    return MB_EINVAL;
  }
  const int B = src->batch;
  if (B == 0) return MB_OK;
  if (!outcomes || !scales) return MB_EINVAL;
  for (int b = 0; b < B; ++b)
    if ((outcomes[b] != 0 && outcomes[b] != 1) || !std::isfinite(scales[b])) {
      set_error("sample %d: outcome must be 0 or 1 and the scale finite", b);
      return MB_EINVAL;
    }
  int* d_out = nullptr;
  double* d_sc = nullptr;
  int rc = dev_alloc((void**)&d_out, sizeof(int) * B);
  if (!rc) rc = dev_alloc((void**)&d_sc, sizeof(double) * B);
  cudaStream_t st = g_ctx.stream;
  if (!rc) {
    cudaMemcpyAsync(d_out, outcomes, sizeof(int) * B, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(d_sc, scales, sizeof(double) * B, cudaMemcpyHostToDevice, st);
    const int64_t work = (int64_t(1) << (src->n - 1)) * B;
    k_remove_qubit<<<grid_for(work, 256), 256, 0, st>>>(src->d, dst->d, src->n, qubit, d_out, d_sc, B);
    ++launch_counter();
    if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess) {
      set_error("remove qubit failed");
      rc = MB_EDEVICE;
    }
  }
  dev_free(d_out);
  dev_free(d_sc);
  return rc;
}

extern "C" int mb_scale_samples(mb_state s, const double* scales) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (int rc = check_init()) return rc;
  if (int rc = check_not_capturing("mb_scale_samples")) return rc;
  if (!s || (!scales && s->batch)) return MB_EINVAL;
  for (int b = 0; b < s->batch; ++b)
    if (!std::isfinite(scales[b])) {
      set_error("scales must be finite");
      return MB_EINVAL;
    }
  if (s->batch == 0) return MB_OK;
  double* d = nullptr;
  int rc = dev_alloc((void**)&d, sizeof(double) * s->batch);
  if (rc) return rc;
  cudaStream_t st = g_ctx.stream;
  cudaMemcpyAsync(d, scales, sizeof(double) * s->batch, cudaMemcpyHostToDevice, st);
  k_scale_samples<<<grid_for(s->elems * s->batch, 256), 256, 0, st>>>(s->d, s->elems, s->batch, d);
  ++launch_counter();
  if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess) {
    set_error("scaling samples failed");
    rc = MB_EDEVICE;
  }
  dev_free(d);
  return rc;
}
