// Partial trace, inner products and fidelities on the device
// (src/observables/partial_trace.jl:11-97, src/states/state_vector.jl:93,
// src/states/density_matrix.jl:129-130, src/states/batch_*.jl fidelity).
//
// partial_tr keeps the remaining qubits in their original order as the low bits of the result
// and sums over the traced ones (_partial_tr_impl): for a density matrix
//   r[a, c] = sum_t rho[(a, t), (c, t)],
// for a pure state r = V V' with V[a, t] = psi[(a, t)]. One thread owns one entry of r and
// loops over t in a fixed order, so the sum is deterministic. Inner products and <y|rho|y>
// reduce per sample in two deterministic stages (per-block partials, then one block per sample).
#include <cmath>
#include <vector>

#include "internal.h"

namespace mb {
namespace {

constexpr int kRThreads = 256;

struct Split {
  int m, k;
  int keep[32];    // remaining qubits, ascending
  int trace[32];   // traced qubits, ascending
};

__device__ __forceinline__ int64_t deposit(int64_t x, int nb, const int* bits) {
  int64_t r = 0;
  for (int j = 0; j < nb; ++j) r |= ((x >> j) & 1) << bits[j];
  return r;
}

__global__ void k_partial_trace(const double2* __restrict__ in, double2* __restrict__ out, int n, int is_dm,
                                const Split sp, int nsamples) {
  const int64_t dm_out = int64_t(1) << sp.m;
  const int64_t per = dm_out * dm_out;
  const int64_t total = per * nsamples;
  const int64_t in_elems = is_dm ? (int64_t(1) << (2 * n)) : (int64_t(1) << n);
  const int64_t dim = int64_t(1) << n;
  const int64_t nt = int64_t(1) << sp.k;
  for (int64_t g = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; g < total; g += int64_t(gridDim.x) * blockDim.x) {
    const int b = int(g / per);
    const int64_t e = g - int64_t(b) * per;
    const int64_t a = e % dm_out, c = e / dm_out;
    const int64_t ra = deposit(a, sp.m, sp.keep), rc = deposit(c, sp.m, sp.keep);
    const double2* s = in + int64_t(b) * in_elems;
    double re = 0.0, im = 0.0;
    for (int64_t t = 0; t < nt; ++t) {
      const int64_t rt = deposit(t, sp.k, sp.trace);
      if (is_dm) {
        const double2 x = s[(ra | rt) + (rc | rt) * dim];
        re += x.x;
        im += x.y;
      } else {
        const double2 u = s[ra | rt], v = s[rc | rt];   // u * conj(v)
        re += u.x * v.x + u.y * v.y;
        im += u.y * v.x - u.x * v.y;
      }
    }
    out[int64_t(b) * per + e] = make_double2(re, im);
  }
}

// Stage 1 of <x|y> (conj on x) or <y|rho|y>: block g of sample b sums a strided range.
__global__ void __launch_bounds__(kRThreads) k_pair_partials(const double2* __restrict__ x, const double2* __restrict__ y,
                                                             int n, int sandwich, int G, double2* __restrict__ part) {
  const int b = blockIdx.y;
  const int64_t dim = int64_t(1) << n;
  const int64_t count = sandwich ? dim * dim : dim;
  const double2* xs = x + int64_t(b) * count;
  const double2* ys = y + int64_t(b) * dim;
  double re = 0.0, im = 0.0;
  for (int64_t i = int64_t(blockIdx.x) * kRThreads + threadIdx.x; i < count; i += int64_t(G) * kRThreads) {
    if (sandwich) {
      // rho[r, c] at r + c*dim contributes conj(y_r) rho[r, c] y_c
      const int64_t r = i & (dim - 1), c = i >> n;
      const double2 rho = xs[i], yr = ys[r], yc = ys[c];
      const double2 t = make_double2(rho.x * yc.x - rho.y * yc.y, rho.x * yc.y + rho.y * yc.x);
      re += yr.x * t.x + yr.y * t.y;
      im += yr.x * t.y - yr.y * t.x;
    } else {
      const double2 u = xs[i], v = ys[i];
      re += u.x * v.x + u.y * v.y;
      im += u.x * v.y - u.y * v.x;
    }
  }
  __shared__ double sre[kRThreads], sim[kRThreads];
  sre[threadIdx.x] = re;
  sim[threadIdx.x] = im;
  __syncthreads();
  for (int w = kRThreads / 2; w > 0; w >>= 1) {
    if (int(threadIdx.x) < w) {
      sre[threadIdx.x] += sre[threadIdx.x + w];
      sim[threadIdx.x] += sim[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) part[int64_t(b) * G + blockIdx.x] = make_double2(sre[0], sim[0]);
}

__global__ void k_pair_finish(const double2* __restrict__ part, int G, double2* __restrict__ out) {
  if (threadIdx.x != 0) return;
  double re = 0.0, im = 0.0;
  for (int g = 0; g < G; ++g) {
    re += part[int64_t(blockIdx.x) * G + g].x;
    im += part[int64_t(blockIdx.x) * G + g].y;
  }
  out[blockIdx.x] = make_double2(re, im);
}

bool is_dm_kind(int kind) { return kind == MB_DENSITY || kind == MB_BATCH_DENSITY; }

int pair_reduce(const double2* x, const double2* y, int n, int sandwich, int B, double* host_out) {
  const int64_t dim = int64_t(1) << n;
  const int64_t count = sandwich ? dim * dim : dim;
  const int G = int(std::max<int64_t>(1, std::min<int64_t>((count + kRThreads - 1) / kRThreads,
                                                          std::max<int64_t>(1, int64_t(g_ctx.sm_count) * 8 / B))));
  double2* part = nullptr;
  double2* res = nullptr;
  int rc = dev_alloc((void**)&part, sizeof(double2) * size_t(G) * B);
  if (!rc) rc = dev_alloc((void**)&res, sizeof(double2) * B);
  cudaStream_t st = g_ctx.stream;
  if (!rc) {
    k_pair_partials<<<dim3(G, B), kRThreads, 0, st>>>(x, y, n, sandwich, G, part);
    k_pair_finish<<<B, 32, 0, st>>>(part, G, res);
    launch_counter() += 2;
    cudaMemcpyAsync(host_out, res, sizeof(double2) * B, cudaMemcpyDeviceToHost, st);
    if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess) {
      set_error("reduction failed");
      rc = MB_EDEVICE;
    }
  }
  dev_free(part);
  dev_free(res);
  return rc;
}

}  // namespace
}  // namespace mb

using namespace mb;

extern "C" int mb_partial_trace(mb_state in, const int* sites, int k, mb_state out) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (int rc = check_init()) return rc;
  if (int rc = check_not_capturing("mb_partial_trace")) return rc;
  if (!in || !out || in == out || k < 1 || (k && !sites)) return MB_EINVAL;
  const int n = in->n;
  if (k >= n) {
    set_error("trace out between 1 and n-1 qubits (the full trace is a scalar)");
    return MB_EINVAL;
  }
  Split sp{};
  sp.m = n - k;
  sp.k = k;
  bool traced[64] = {false};
  for (int j = 0; j < k; ++j) {
    if (sites[j] < 0 || sites[j] >= n) {
      set_error("site out of range.");
      return MB_EINVAL;
    }
    if (traced[sites[j]]) {
      set_error("duplicate sites not allowed.");
      return MB_EINVAL;
    }
    traced[sites[j]] = true;
  }
  for (int q = 0, a = 0, t = 0; q < n; ++q) {
    if (traced[q]) sp.trace[t++] = q;
    else sp.keep[a++] = q;
  }
  const bool batch_in = in->kind == MB_BATCH_PURE || in->kind == MB_BATCH_DENSITY;
  const int want_kind = batch_in ? MB_BATCH_DENSITY : MB_DENSITY;
  if (out->kind != want_kind || out->n != sp.m || out->batch != in->batch) {
    set_error("partial trace output must be a %s of %d qubits and the input's batch size",
              batch_in ? "BatchDensityMatrix" : "DensityMatrix", sp.m);
    return MB_EINVAL;
  }
  if (in->batch == 0) return MB_OK;
  const int64_t work = (int64_t(1) << (2 * sp.m)) * in->batch;
  k_partial_trace<<<grid_for(work, 256), 256, 0, g_ctx.stream>>>(in->d, out->d, n, is_dm_kind(in->kind) ? 1 : 0, sp,
                                                                  in->batch);
  MB_LAUNCHED();
  MB_CHECK_CUDA(cudaStreamSynchronize(g_ctx.stream));
  return MB_OK;
}

extern "C" int mb_inner(mb_state x, mb_state y, double* out) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (int rc = check_init()) return rc;
  if (int rc = check_not_capturing("mb_inner")) return rc;
  if (!x || !y || !out) return MB_EINVAL;
  if (is_dm_kind(x->kind) || is_dm_kind(y->kind) || x->n != y->n || x->batch != y->batch) {
    set_error("inner products need two pure states of the same size and batch");
    return MB_EINVAL;
  }
  if (x->batch == 0) return MB_OK;
  return pair_reduce(x->d, y->d, x->n, 0, x->batch, out);
}

extern "C" int mb_sandwich(mb_state rho, mb_state y, double* out) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (int rc = check_init()) return rc;
  if (int rc = check_not_capturing("mb_sandwich")) return rc;
  if (!rho || !y || !out) return MB_EINVAL;
  if (!is_dm_kind(rho->kind) || is_dm_kind(y->kind) || rho->n != y->n || rho->batch != y->batch) {
    set_error("<y|rho|y> needs a density matrix and a pure state of the same size and batch");
    return MB_EINVAL;
  }
  if (rho->batch == 0) return MB_OK;
  return pair_reduce(rho->d, y->d, rho->n, 1, rho->batch, out);
}

extern "C" int mb_state_extract(mb_state src, int index, mb_state dst) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (int rc = check_init()) return rc;
  if (!src || !dst || index < 0 || index >= src->batch) return MB_EINVAL;
  const bool ok = ((src->kind == MB_BATCH_PURE && dst->kind == MB_PURE) ||
                   (src->kind == MB_BATCH_DENSITY && dst->kind == MB_DENSITY)) && dst->n == src->n;
  if (!ok) {
    set_error("extract needs a batch source and a single state of the same kind and size");
    return MB_EINVAL;
  }
  MB_CHECK_CUDA(cudaMemcpyAsync(dst->d, src->d + int64_t(index) * src->elems, sizeof(double2) * src->elems,
                                cudaMemcpyDeviceToDevice, g_ctx.stream));
  MB_CHECK_CUDA(cudaStreamSynchronize(g_ctx.stream));
  return MB_OK;
}

extern "C" int mb_state_broadcast(mb_state src, mb_state dst) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (int rc = check_init()) return rc;
  if (!src || !dst) return MB_EINVAL;
  const bool ok = ((src->kind == MB_PURE && dst->kind == MB_BATCH_PURE) ||
                   (src->kind == MB_DENSITY && dst->kind == MB_BATCH_DENSITY)) && dst->n == src->n;
  if (!ok) {
    set_error("broadcast needs a single source and a batch destination of the same kind and size");
    return MB_EINVAL;
  }
  for (int b = 0; b < dst->batch; ++b)
    MB_CHECK_CUDA(cudaMemcpyAsync(dst->d + int64_t(b) * dst->elems, src->d, sizeof(double2) * src->elems,
                                  cudaMemcpyDeviceToDevice, g_ctx.stream));
  MB_CHECK_CUDA(cudaStreamSynchronize(g_ctx.stream));
  return MB_OK;
}

extern "C" int mb_state_tile(mb_state src, int copies, mb_state dst) {
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (int rc = check_init()) return rc;
  if (!src || !dst || copies < 0) return MB_EINVAL;
  if (src->kind != dst->kind || src->kind < MB_BATCH_PURE || dst->n != src->n ||
      int64_t(dst->batch) != int64_t(src->batch) * copies) {
    set_error("tile needs batch states of one kind and size, the destination holding `copies` copies of the source");
    return MB_EINVAL;
  }
  const size_t bytes = sizeof(double2) * size_t(src->elems) * src->batch;
  for (int c = 0; c < copies; ++c)
    MB_CHECK_CUDA(cudaMemcpyAsync(reinterpret_cast<char*>(dst->d) + bytes * c, src->d, bytes, cudaMemcpyDeviceToDevice,
                                  g_ctx.stream));
  MB_CHECK_CUDA(cudaStreamSynchronize(g_ctx.stream));
  return MB_OK;
}
