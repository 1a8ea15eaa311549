// Expectation of one local operator without any device allocation.
//
// Some callers cannot allocate device memory: code that runs inside a pre-planned memory
// pool with every byte already assigned (a serving process that sized its HBM budget up
// front), host runtimes that must not call cudaMalloc/cudaFree on their latency-critical
// path because those calls synchronise the device, and plug-ins that may only touch memory
// their host hands them. mb_expect_local_noalloc serves them: the caller passes the state
// (device memory it owns) and receives <psi|M|psi> per sample; the partial sums of the
// reduction live in the file-scope array below instead of a workspace from mb_init.
//
// The array holds 82,560 bytes and lives on every GPU that loads this library until the process
// exits. All calls share it, and each call keeps its contents until the next call: two
// calls that overlap on the GPU (different streams or threads) race on it and must be
// serialised by the caller. The array's device address is looked up on the first call on each
// device and kept for the life of the process, so the entry point must not be used after the
// caller resets that device (cudaDeviceReset), which invalidates the address.
#include <cmath>
#include <mutex>

#include "common.cuh"

namespace mb {
namespace {

constexpr int kNaMaxSamples = 32;        // samples per call
constexpr int kNaBlocksPerSample = 160;  // reduction blocks per sample
constexpr int kNaMaxK = 3;               // operator on at most 3 qubits (8x8 matrix)
constexpr int kNaThreads = 256;

// Layout of the static scratch: partial sums, per-sample results, block counters.
constexpr size_t kNaPartialBytes = sizeof(double2) * kNaMaxSamples * kNaBlocksPerSample;
constexpr size_t kNaResultBytes = sizeof(double2) * kNaMaxSamples;
constexpr size_t kNaCounterBytes = sizeof(unsigned) * kNaMaxSamples;
constexpr size_t kNaScratchBytes = kNaPartialBytes + kNaResultBytes + kNaCounterBytes;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNaScratchBytes];

struct NaMatrix {
  double2 m[(1 << kNaMaxK) * (1 << kNaMaxK)];
  int64_t off[1 << kNaMaxK];
  int k;
  int pos[kNaMaxK];
};

__global__ void __launch_bounds__(kNaThreads) k_expect_noalloc(const double2* __restrict__ v, int64_t dim,
                                                              const NaMatrix mat, unsigned char* scratch) {
  double2* partials = reinterpret_cast<double2*>(scratch);
  double2* results = reinterpret_cast<double2*>(scratch + kNaPartialBytes);
  unsigned* counters = reinterpret_cast<unsigned*>(scratch + kNaPartialBytes + kNaResultBytes);
  const int b = blockIdx.y, G = gridDim.x, k = mat.k, d = 1 << k;
  const double2* vs = v + int64_t(b) * dim;
  const int64_t nblk = dim >> k;
  double2 acc = cz();
  for (int64_t j = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; j < nblk; j += int64_t(G) * blockDim.x) {
    const int64_t base = insert_zeros(j, k, mat.pos);
    double2 x[1 << kNaMaxK];
    for (int a = 0; a < d; ++a) x[a] = vs[base + mat.off[a]];
    for (int r = 0; r < d; ++r) {
      double2 mv = cz();
      for (int c = 0; c < d; ++c) mv = cfma(mat.m[r + c * d], x[c], mv);
      acc = cfma_conj(x[r], mv, acc);
    }
  }
  // block sum, then the last block of the sample sums the partials in order
  __shared__ double2 wsum[kNaThreads / 32];
  __shared__ bool last;
  for (int o = 16; o > 0; o >>= 1) {
    acc.x += __shfl_down_sync(0xffffffffu, acc.x, o);
    acc.y += __shfl_down_sync(0xffffffffu, acc.y, o);
  }
  if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double2 s = cz();
    for (int w = 0; w < kNaThreads / 32; ++w) s = cadd(s, wsum[w]);
    partials[int64_t(b) * kNaBlocksPerSample + blockIdx.x] = s;
    __threadfence();
    last = atomicAdd(&counters[b], 1u) == unsigned(G - 1);
  }
  __syncthreads();
  if (last && threadIdx.x == 0) {
    double2 s = cz();
    for (int g = 0; g < G; ++g) s = cadd(s, __ldcg(&partials[int64_t(b) * kNaBlocksPerSample + g]));
    results[b] = s;
    counters[b] = 0;
  }
}

std::mutex g_na_mu;
void* g_na_addr[64] = {nullptr};

}  // namespace
}  // namespace mb

using namespace mb;

extern "C" int mb_expect_local_noalloc(const double* state_dev, int n, int nsamples, int k, const int* positions,
                                       const double* matrix, double* out, void* stream) {
  if (!state_dev || !positions || !matrix || !out) {
    set_error("mb_expect_local_noalloc: null argument");
    return MB_EINVAL;
  }
  if (n < 1 || n > 34) {
    set_error("mb_expect_local_noalloc: %d qubits outside 1..34", n);
    return MB_EINVAL;
  }
  if (nsamples < 1 || nsamples > kNaMaxSamples) {
    set_error("mb_expect_local_noalloc: %d samples exceed the static scratch (at most %d per call)", nsamples,
              kNaMaxSamples);
    return MB_EINVAL;
  }
  if (k < 1 || k > kNaMaxK || k > n) {
    set_error("mb_expect_local_noalloc: operator on %d qubits; at most %d supported", k, kNaMaxK);
    return MB_EINVAL;
  }
  if ((reinterpret_cast<uintptr_t>(state_dev) & 15) != 0) {
    set_error("mb_expect_local_noalloc: state must be 16-byte aligned");
    return MB_EINVAL;
  }
  NaMatrix mat{};
  mat.k = k;
  for (int j = 0; j < k; ++j) {
    if (positions[j] < 0 || positions[j] >= n) {
      set_error("mb_expect_local_noalloc: position %d out of range", positions[j]);
      return MB_EINVAL;
    }
    for (int q = 0; q < j; ++q)
      if (positions[q] == positions[j]) {
        set_error("mb_expect_local_noalloc: positions must be distinct");
        return MB_EINVAL;
      }
  }
  // Sort the positions and permute the matrix like ordered_mat.
  int seq[kNaMaxK] = {0, 1, 2};
  for (int a = 0; a < k; ++a)
    for (int b2 = a + 1; b2 < k; ++b2)
      if (positions[seq[b2]] < positions[seq[a]]) { int t = seq[a]; seq[a] = seq[b2]; seq[b2] = t; }
  const int d = 1 << k;
  int perm[1 << kNaMaxK];
  for (int ap = 0; ap < d; ++ap) {
    int a = 0;
    for (int j = 0; j < k; ++j)
      if ((ap >> j) & 1) a |= 1 << seq[j];
    perm[ap] = a;
  }
  for (int j = 0; j < k; ++j) mat.pos[j] = positions[seq[j]];
  for (int ap = 0; ap < d; ++ap) {
    int64_t o = 0;
    for (int j = 0; j < k; ++j)
      if ((ap >> j) & 1) o |= int64_t(1) << mat.pos[j];
    mat.off[ap] = o;
    for (int bp = 0; bp < d; ++bp) {
      const int a = perm[ap], bb = perm[bp];
      const double re = matrix[2 * (a + bb * d)], im = matrix[2 * (a + bb * d) + 1];
      if (!std::isfinite(re) || !std::isfinite(im)) {
        set_error("mb_expect_local_noalloc: matrix must be finite");
        return MB_EINVAL;
      }
      mat.m[ap + bp * d] = make_double2(re, im);
    }
  }
  // Set-up, once per device with that device current: the device address of the scratch.
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= 64) {
    set_error("mb_expect_local_noalloc: no current CUDA device (%s)", cudaGetErrorString(e));
    return MB_EDEVICE;
  }
  void* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_na_mu);
    if (!g_na_addr[dev]) {
      e = cudaGetSymbolAddress(&g_na_addr[dev], g_noalloc_scratch);
      if (e != cudaSuccess) {
        g_na_addr[dev] = nullptr;
        set_error("mb_expect_local_noalloc: scratch address lookup failed: %s", cudaGetErrorString(e));
        return MB_EDEVICE;
      }
    }
    scratch = g_na_addr[dev];
  }
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  unsigned char* sc = static_cast<unsigned char*>(scratch);
  // The block counters must start at zero.
  e = cudaMemsetAsync(sc + kNaPartialBytes + kNaResultBytes, 0, kNaCounterBytes, st);
  if (e != cudaSuccess) {
    set_error("mb_expect_local_noalloc: %s", cudaGetErrorString(e));
    return MB_EDEVICE;
  }
  const int64_t dim = int64_t(1) << n;
  int64_t blocks = ((dim >> k) + kNaThreads - 1) / kNaThreads;
  if (blocks > kNaBlocksPerSample) blocks = kNaBlocksPerSample;
  if (blocks < 1) blocks = 1;
  k_expect_noalloc<<<dim3(unsigned(blocks), unsigned(nsamples)), kNaThreads, 0, st>>>(
      reinterpret_cast<const double2*>(state_dev), dim, mat, sc);
  e = cudaGetLastError();
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(out, sc + kNaPartialBytes, sizeof(double2) * nsamples, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    set_error("mb_expect_local_noalloc: %s", cudaGetErrorString(e));
    return MB_EDEVICE;
  }
  ++launch_counter();
  return MB_OK;
}
