// Plain per-gate sweeps, reductions, readout and parameter binding (sm_100a).
//
// These are the direct B200 equivalents of the reference's CPU kernels:
//   dense gate sweep       src/backends/cpu/gates/serial_short_range.jl:2-71,
//                          threaded_long_range.jl:3-132      -> k_dense<K>
//   diagonal / permutation src/backends/cpu/gates/specific/*.jl -> k_diag, k_monomial
//   expectation            src/backends/cpu/expectations/threaded*.jl -> k_cross_dense<K>
//   density expectation    src/backends/cpu/expectations/density_matrix_serial.jl -> k_dm_trace<K>
//   observable action      src/backends/cpu/operators/generic.jl:12-24 -> k_obs_apply<K>
//   probabilities          src/execution/probabilities.jl:42-105 -> k_marginal
// One thread owns one block of 2^K amplitudes that share all non-gate bits; consecutive
// threads own consecutive blocks, so the loads of a warp are coalesced double2 (16 B)
// accesses whenever the gate bits are not the lowest ones.
#include <cstdarg>

#include "family.cuh"
#include "kernels.h"

namespace mb {

namespace {

constexpr int kBlock = 256;

template <int D>
__device__ __forceinline__ void load_matrix(double2* sm, const double2* m, int mode) {
  for (int e = threadIdx.x; e < D * D; e += blockDim.x) sm[e] = mat_at(m, D, e % D, e / D, mode);
}

template <int K>
__device__ __forceinline__ void load_offsets(int64_t* soff, const Pos& pos) {
  constexpr int D = 1 << K;
  for (int a = threadIdx.x; a < D; a += blockDim.x) {
    int64_t o = 0;
#pragma unroll
    for (int j = 0; j < K; ++j)
      if ((a >> j) & 1) o |= int64_t(1) << pos.p[j];
    soff[a] = o;
  }
}

template <int K>
__global__ void __launch_bounds__(kBlock) k_dense(double2* __restrict__ v, int64_t elems, Pos pos,
                                                   const double2* __restrict__ mats, int64_t mstride, int mode) {
  constexpr int D = 1 << K;
  __shared__ double2 sm[D * D];
  __shared__ int64_t soff[D];
  const int b = blockIdx.y;
  load_matrix<D>(sm, mats + b * mstride, mode);
  load_offsets<K>(soff, pos);
  __syncthreads();
  double2* vs = v + int64_t(b) * elems;
  const int64_t nblk = elems >> K;
  for (int64_t j = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; j < nblk; j += int64_t(gridDim.x) * blockDim.x) {
    const int64_t base = insert_zeros(j, K, pos.p);
    double2 in[D];
#pragma unroll
    for (int a = 0; a < D; ++a) in[a] = vs[base + soff[a]];
#pragma unroll
    for (int r = 0; r < D; ++r) {
      double2 acc = cmul(sm[r], in[0]);
#pragma unroll
      for (int c = 1; c < D; ++c) acc = cfma(sm[r + c * D], in[c], acc);
      vs[base + soff[r]] = acc;
    }
  }
}

template <int K>
__global__ void __launch_bounds__(kBlock) k_diag(double2* __restrict__ v, int64_t elems, Pos pos,
                                                  const double2* __restrict__ mats, int64_t mstride, int mode,
                                                  uint32_t active) {
  constexpr int D = 1 << K;
  __shared__ double2 sd[D];
  __shared__ int64_t soff[D];
  const int b = blockIdx.y;
  for (int a = threadIdx.x; a < D; a += blockDim.x) sd[a] = mat_at(mats + b * mstride, D, a, a, mode);
  load_offsets<K>(soff, pos);
  __syncthreads();
  double2* vs = v + int64_t(b) * elems;
  const int64_t nblk = elems >> K;
  for (int64_t j = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; j < nblk; j += int64_t(gridDim.x) * blockDim.x) {
    const int64_t base = insert_zeros(j, K, pos.p);
#pragma unroll
    for (int a = 0; a < D; ++a)
      if ((active >> a) & 1) {
        double2 x = vs[base + soff[a]];
        vs[base + soff[a]] = cmul(sd[a], x);
      }
  }
}

struct Sigma {
  int n;          // active entries
  int from[32];   // local index read
  int to[32];     // local index written
};

template <int K>
__global__ void __launch_bounds__(kBlock) k_monomial(double2* __restrict__ v, int64_t elems, Pos pos,
                                                      const double2* __restrict__ mats, int64_t mstride,
                                                      int mode, Sigma sg) {
  constexpr int D = 1 << K;
  __shared__ double2 sph[D];
  __shared__ int64_t soff[D];
  const int b = blockIdx.y;
  for (int e = threadIdx.x; e < sg.n; e += blockDim.x)
    sph[e] = mat_at(mats + b * mstride, D, sg.to[e], sg.from[e], mode);
  load_offsets<K>(soff, pos);
  __syncthreads();
  double2* vs = v + int64_t(b) * elems;
  const int64_t nblk = elems >> K;
  for (int64_t j = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; j < nblk; j += int64_t(gridDim.x) * blockDim.x) {
    const int64_t base = insert_zeros(j, K, pos.p);
    double2 x[D];
#pragma unroll
    for (int e = 0; e < D; ++e)
      if (e < sg.n) x[e] = vs[base + soff[sg.from[e]]];
#pragma unroll
    for (int e = 0; e < D; ++e)
      if (e < sg.n) vs[base + soff[sg.to[e]]] = cmul(sph[e], x[e]);
  }
}

__global__ void k_set_basis(double2* v, int64_t elems, int64_t index) {
  const int b = blockIdx.y;
  double2* vs = v + int64_t(b) * elems;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < elems; i += int64_t(gridDim.x) * blockDim.x)
    vs[i] = make_double2(i == index ? 1.0 : 0.0, 0.0);
}

// rho[r + dim*c] = psi[r] conj(psi[c])
__global__ void k_to_density(const double2* __restrict__ psi, double2* __restrict__ rho, int n) {
  const int b = blockIdx.y;
  const int64_t dim = int64_t(1) << n, elems = dim * dim;
  const double2* p = psi + int64_t(b) * dim;
  double2* r = rho + int64_t(b) * elems;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < elems; i += int64_t(gridDim.x) * blockDim.x) {
    const int64_t row = i & (dim - 1), col = i >> n;
    r[i] = cmul(p[row], cconj(p[col]));
  }
}

__global__ void k_identity_density(double2* rho, int n) {
  const int b = blockIdx.y;
  const int64_t dim = int64_t(1) << n, elems = dim * dim;
  double2* r = rho + int64_t(b) * elems;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < elems; i += int64_t(gridDim.x) * blockDim.x)
    r[i] = make_double2((i & (dim - 1)) == (i >> n) ? 1.0 : 0.0, 0.0);
}

__global__ void k_scale(double2* v, int64_t count, double s) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < count; i += int64_t(gridDim.x) * blockDim.x)
    v[i] = cscale(v[i], s);
}

// ---- block reduction + last-block completion ---------------------------------------------
__device__ __forceinline__ double2 warp_sum(double2 x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    x.x += __shfl_down_sync(0xffffffffu, x.x, o);
    x.y += __shfl_down_sync(0xffffffffu, x.y, o);
  }
  return x;
}

// Reduces `acc` over the block, stores the block partial, and lets the last block of the
// sample (then the last sample) finish the reduction in a fixed order.
__device__ void finish_reduction(double2 acc, double2* partials, unsigned* counters, const ReduceOut& ro) {
  __shared__ double2 warp_part[32];
  __shared__ bool last_block, last_sample;
  const int b = blockIdx.y, nb = gridDim.y, G = gridDim.x;
  acc = warp_sum(acc);
  if ((threadIdx.x & 31) == 0) warp_part[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double2 s = cz();
    for (int w = 0; w < int(blockDim.x >> 5); ++w) s = cadd(s, warp_part[w]);
    partials[int64_t(b) * G + blockIdx.x] = s;
    __threadfence();
    unsigned ticket = atomicAdd(&counters[b], 1u);
    last_block = ticket == unsigned(G - 1);
  }
  __syncthreads();
  if (!last_block) return;
  if (threadIdx.x == 0) {
    double2 s = cz();
    for (int g = 0; g < G; ++g) s = cadd(s, __ldcg(&partials[int64_t(b) * G + g]));
    counters[b] = 0;
    if (ro.out) ro.out[b] = ro.accumulate ? cadd(__ldcg(&ro.out[b]), s) : s;
    // Per-sample results also land in partials[nb * G + b] for the weighted total.
    partials[int64_t(nb) * G + b] = s;
    __threadfence();
    unsigned ticket = atomicAdd(&counters[nb], 1u);
    last_sample = ticket == unsigned(nb - 1);
    if (last_sample) {
      counters[nb] = 0;
      if (ro.grad) {
        double t = 0.0;
        for (int q = 0; q < nb; ++q) {
          double w = ro.weights ? ro.weights[q] : 1.0;
          t += w * __ldcg(&partials[int64_t(nb) * G + q]).x;
        }
        ro.grad[0] += t;
      }
    }
  }
}

template <int K>
__global__ void __launch_bounds__(kBlock) k_cross_dense(const double2* __restrict__ c, const double2* __restrict__ v,
                                                         int64_t elems, Pos pos, const double2* __restrict__ mats,
                                                         int64_t mstride, int mode, double2* partials,
                                                         unsigned* counters, ReduceOut ro) {
  constexpr int D = 1 << K;
  __shared__ double2 sm[D * D];
  __shared__ int64_t soff[D];
  const int b = blockIdx.y;
  load_matrix<D>(sm, mats + b * mstride, mode);
  load_offsets<K>(soff, pos);
  __syncthreads();
  const double2* cs = c + int64_t(b) * elems;
  const double2* vs = v + int64_t(b) * elems;
  const int64_t nblk = elems >> K;
  double2 acc = cz();
  for (int64_t j = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; j < nblk; j += int64_t(gridDim.x) * blockDim.x) {
    const int64_t base = insert_zeros(j, K, pos.p);
    double2 in[D];
#pragma unroll
    for (int a = 0; a < D; ++a) in[a] = vs[base + soff[a]];
#pragma unroll
    for (int r = 0; r < D; ++r) {
      double2 mv = cmul(sm[r], in[0]);
#pragma unroll
      for (int q = 1; q < D; ++q) mv = cfma(sm[r + q * D], in[q], mv);
      acc = cfma_conj(cs[base + soff[r]], mv, acc);
    }
  }
  finish_reduction(acc, partials, counters, ro);
}

// Scalar (zero-qubit) cross product sum conj(c) v.
__global__ void __launch_bounds__(kBlock) k_cross_scalar(const double2* __restrict__ c, const double2* __restrict__ v,
                                                          int64_t elems, const double2* __restrict__ m,
                                                          double2* partials, unsigned* counters, ReduceOut ro) {
  const int b = blockIdx.y;
  const double2 scale = m[0];
  const double2* cs = c + int64_t(b) * elems;
  const double2* vs = v + int64_t(b) * elems;
  double2 acc = cz();
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < elems; i += int64_t(gridDim.x) * blockDim.x)
    acc = cfma_conj(cs[i], vs[i], acc);
  acc = cmul(scale, acc);
  finish_reduction(acc, partials, counters, ro);
}

template <int K>
__global__ void __launch_bounds__(kBlock) k_dm_trace(const double2* __restrict__ rho, int n, Pos pos,
                                                      const double2* __restrict__ m, double2* partials,
                                                      unsigned* counters, ReduceOut ro) {
  constexpr int D = 1 << K;
  __shared__ double2 sm[D * D];
  __shared__ int64_t soff[D];
  const int b = blockIdx.y;
  load_matrix<D>(sm, m, MAT_PLAIN);
  load_offsets<K>(soff, pos);
  __syncthreads();
  const int64_t dim = int64_t(1) << n;
  const double2* r = rho + int64_t(b) * dim * dim;
  const int64_t nblk = dim >> K;
  double2 acc = cz();
  for (int64_t j = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; j < nblk; j += int64_t(gridDim.x) * blockDim.x) {
    const int64_t base = insert_zeros(j, K, pos.p);
#pragma unroll
    for (int a = 0; a < D; ++a)
#pragma unroll
      for (int q = 0; q < D; ++q)  // M[a,q] * rho[base|q, base|a]
        acc = cfma(sm[a + q * D], r[(base + soff[q]) + dim * (base + soff[a])], acc);
  }
  finish_reduction(acc, partials, counters, ro);
}

// s * tr(rho) (the identity key of an observable on a density matrix).
__global__ void __launch_bounds__(kBlock) k_dm_trace0(const double2* __restrict__ rho, int n,
                                                       const double2* __restrict__ m, double2* partials,
                                                       unsigned* counters, ReduceOut ro) {
  const int b = blockIdx.y;
  const int64_t dim = int64_t(1) << n;
  const double2* r = rho + int64_t(b) * dim * dim;
  double2 acc = cz();
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < dim; i += int64_t(gridDim.x) * blockDim.x)
    acc = cadd(acc, r[i + dim * i]);
  acc = cmul(m[0], acc);
  finish_reduction(acc, partials, counters, ro);
}

template <int K>
__global__ void __launch_bounds__(kBlock) k_obs_apply(const double2* __restrict__ in, double2* __restrict__ out,
                                                       int64_t elems, Pos pos, const double2* __restrict__ m,
                                                       int first) {
  constexpr int D = 1 << K;
  __shared__ double2 sm[D * D];
  __shared__ int64_t soff[D];
  const int b = blockIdx.y;
  load_matrix<D>(sm, m, MAT_PLAIN);
  load_offsets<K>(soff, pos);
  __syncthreads();
  const double2* is = in + int64_t(b) * elems;
  double2* os = out + int64_t(b) * elems;
  const int64_t nblk = elems >> K;
  for (int64_t j = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; j < nblk; j += int64_t(gridDim.x) * blockDim.x) {
    const int64_t base = insert_zeros(j, K, pos.p);
    double2 x[D];
#pragma unroll
    for (int a = 0; a < D; ++a) x[a] = is[base + soff[a]];
#pragma unroll
    for (int r = 0; r < D; ++r) {
      double2 acc = first ? cz() : os[base + soff[r]];
#pragma unroll
      for (int q = 0; q < D; ++q) acc = cfma(sm[r + q * D], x[q], acc);
      os[base + soff[r]] = acc;
    }
  }
}

__global__ void k_obs_scalar(const double2* __restrict__ in, double2* __restrict__ out, int64_t count,
                             const double2* __restrict__ m, int first) {
  const double2 s = m[0];
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < count; i += int64_t(gridDim.x) * blockDim.x)
    out[i] = first ? cmul(s, in[i]) : cfma(s, in[i], out[i]);
}

struct Readout {
  int nq;
  int q[30];
};

// Marginal histogram in shared memory (nq <= 12), merged into out with double atomics.
__global__ void __launch_bounds__(kBlock) k_marginal_small(const double2* __restrict__ v, int n, int is_dm,
                                                            Readout ro, double* out, unsigned* flags, double tol) {
  extern __shared__ double hist[];
  const int b = blockIdx.y;
  const int M = 1 << ro.nq;
  const int64_t dim = int64_t(1) << n;
  const int64_t elems = is_dm ? dim * dim : dim;
  const double2* vs = v + int64_t(b) * elems;
  for (int r = threadIdx.x; r < M; r += blockDim.x) hist[r] = 0.0;
  __syncthreads();
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < dim; i += int64_t(gridDim.x) * blockDim.x) {
    double p;
    if (is_dm) {
      double2 x = vs[i + dim * i];
      if (fabs(x.y) > tol) atomicOr(&flags[0], 1u);
      if (x.x < -tol) atomicOr(&flags[1], 1u);
      p = x.x;
    } else {
      double2 x = vs[i];
      p = x.x * x.x + x.y * x.y;
    }
    int r = 0;
    for (int j = 0; j < ro.nq; ++j) r |= int((i >> ro.q[j]) & 1) << j;
    atomicAdd(&hist[r], p);
  }
  __syncthreads();
  for (int r = threadIdx.x; r < M; r += blockDim.x)
    if (hist[r] != 0.0) atomicAdd(&out[int64_t(b) * M + r], hist[r]);
}

__global__ void __launch_bounds__(kBlock) k_marginal_large(const double2* __restrict__ v, int n, int is_dm,
                                                            Readout ro, double* out, unsigned* flags, double tol,
                                                            int identity) {
  const int b = blockIdx.y;
  const int64_t M = int64_t(1) << ro.nq;
  const int64_t dim = int64_t(1) << n;
  const int64_t elems = is_dm ? dim * dim : dim;
  const double2* vs = v + int64_t(b) * elems;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < dim; i += int64_t(gridDim.x) * blockDim.x) {
    double p;
    if (is_dm) {
      double2 x = vs[i + dim * i];
      if (fabs(x.y) > tol) atomicOr(&flags[0], 1u);
      if (x.x < -tol) atomicOr(&flags[1], 1u);
      p = x.x;
    } else {
      double2 x = vs[i];
      p = x.x * x.x + x.y * x.y;
    }
    if (identity) {
      out[int64_t(b) * M + i] = p;
    } else {
      int64_t r = 0;
      for (int j = 0; j < ro.nq; ++j) r |= ((i >> ro.q[j]) & 1) << j;
      atomicAdd(&out[int64_t(b) * M + r], p);
    }
  }
}

// ---- parameter binding --------------------------------------------------------------------
// (family_matrix and bind_record: family.cuh, shared with the host-side lowering check)
__global__ void k_bind(const BindRec* __restrict__ recs, int nrecs, const double* __restrict__ theta, int nslots,
                       int rows, double2* table, int64_t stride) {
  const int64_t idx = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (idx >= int64_t(nrecs) * rows) return;
  const int row = int(idx / nrecs), q = int(idx % nrecs);
  const BindRec rc = recs[q];
  const double t = rc.slot >= 0 ? theta[int64_t(row) * nslots + rc.slot] : rc.value;
  bind_record(rc, t, table, table + int64_t(row) * stride);
}

}  // namespace

// ---------------------------------------------------------------------------------------------
// Launchers
// ---------------------------------------------------------------------------------------------
#define MB_DISPATCH_K(K, CALL) \
  switch (K) {                 \
    case 1: { constexpr int KK = 1; CALL; } break; \
    case 2: { constexpr int KK = 2; CALL; } break; \
    case 3: { constexpr int KK = 3; CALL; } break; \
    case 4: { constexpr int KK = 4; CALL; } break; \
    case 5: { constexpr int KK = 5; CALL; } break; \
    default: set_error("unsupported local operator size %d", K); return MB_EUNSUPPORTED; \
  }

static dim3 sample_grid(int64_t work, int nsamples) {
  int64_t per = (int64_t(148) * 8 + nsamples - 1) / nsamples;
  if (per < 1) per = 1;
  return dim3(grid_for(work, kBlock, per), nsamples);
}

int launch_dense(double2* v, int64_t elems, int nsamples, const Pos& pos, const double2* mats, int64_t mstride,
                 int mode, cudaStream_t st) {
  if (nsamples <= 0 || elems == 0) return MB_OK;
  dim3 g = sample_grid(elems >> pos.k, nsamples);
  {
    ProfScope ps("k_dense", 32.0 * elems * nsamples, st, 8.0 * (1 << pos.k) * elems * nsamples);
    MB_DISPATCH_K(pos.k, (k_dense<KK><<<g, kBlock, 0, st>>>(v, elems, pos, mats, mstride, mode)));
  }
  MB_LAUNCHED();
  return MB_OK;
}

int launch_diag(double2* v, int64_t elems, int nsamples, const Pos& pos, const double2* mats, int64_t mstride,
                int mode, uint32_t active, cudaStream_t st) {
  if (nsamples <= 0 || elems == 0 || active == 0) return MB_OK;
  dim3 g = sample_grid(elems >> pos.k, nsamples);
  {
    ProfScope ps("k_diag", 32.0 * elems * nsamples * __builtin_popcount(active) / (1 << pos.k), st);
    MB_DISPATCH_K(pos.k, (k_diag<KK><<<g, kBlock, 0, st>>>(v, elems, pos, mats, mstride, mode, active)));
  }
  MB_LAUNCHED();
  return MB_OK;
}

int launch_monomial(double2* v, int64_t elems, int nsamples, const Pos& pos, const double2* mats, int64_t mstride,
                    int mode, const int* sigma, int d, cudaStream_t st) {
  if (nsamples <= 0 || elems == 0) return MB_OK;
  Sigma sg{};
  // sigma[a] < 0 marks an entry the caller found unchanged (fixed point with phase 1).
  for (int a = 0; a < d; ++a)
    if (sigma[a] >= 0) { sg.from[sg.n] = a; sg.to[sg.n] = sigma[a]; ++sg.n; }
  if (sg.n == 0) return MB_OK;
  dim3 g = sample_grid(elems >> pos.k, nsamples);
  {
    ProfScope ps("k_monomial", 32.0 * elems * nsamples * sg.n / (1 << pos.k), st);
    MB_DISPATCH_K(pos.k, (k_monomial<KK><<<g, kBlock, 0, st>>>(v, elems, pos, mats, mstride, mode, sg)));
  }
  MB_LAUNCHED();
  return MB_OK;
}

int launch_set_basis(double2* v, int64_t elems, int nsamples, int64_t index, cudaStream_t st) {
  if (nsamples <= 0) return MB_OK;
  k_set_basis<<<sample_grid(elems, nsamples), kBlock, 0, st>>>(v, elems, index);
  MB_LAUNCHED();
  return MB_OK;
}

int launch_to_density(const double2* psi, double2* rho, int n, int nsamples, cudaStream_t st) {
  if (nsamples <= 0) return MB_OK;
  k_to_density<<<sample_grid(int64_t(1) << (2 * n), nsamples), kBlock, 0, st>>>(psi, rho, n);
  MB_LAUNCHED();
  return MB_OK;
}

int launch_identity_density(double2* rho, int n, int nsamples, cudaStream_t st) {
  if (nsamples <= 0) return MB_OK;
  k_identity_density<<<sample_grid(int64_t(1) << (2 * n), nsamples), kBlock, 0, st>>>(rho, n);
  MB_LAUNCHED();
  return MB_OK;
}

int launch_scale(double2* v, int64_t count, double s, cudaStream_t st) {
  if (count <= 0) return MB_OK;
  k_scale<<<grid_for(count, kBlock), kBlock, 0, st>>>(v, count, s);
  MB_LAUNCHED();
  return MB_OK;
}

static int reduce_grid(int64_t work, int nsamples, const ReduceWs& ws, int slot, dim3* g) {
  int64_t cap_per = (ws.capacity / (nsamples + 1)) - 1;
  int64_t per = std::min<int64_t>((int64_t(148) * 4 + nsamples - 1) / nsamples, cap_per);
  if (per < 1 || nsamples + 1 > ws.ncounters) {
    set_error("reduction workspace too small for %d samples", nsamples);
    return MB_EUNSUPPORTED;
  }
  (void)slot;
  *g = dim3(grid_for(work, kBlock, per), nsamples);
  return MB_OK;
}

int launch_cross_dense(const double2* c, const double2* v, int64_t elems, int nsamples, const Pos& pos,
                       const double2* m, int64_t mstride, int mode, const ReduceWs& ws, int slot,
                       const ReduceOut& ro, cudaStream_t st) {
  if (nsamples <= 0) return MB_OK;
  dim3 g;
  int rc = reduce_grid(elems >> pos.k, nsamples, ws, slot, &g);
  if (rc) return rc;
  if (pos.k == 0) {
    k_cross_scalar<<<g, kBlock, 0, st>>>(c, v, elems, m, ws.partials, ws.counters, ro);
  } else {
    ProfScope ps("k_cross_dense", (c == v ? 16.0 : 32.0) * elems * nsamples, st);
    MB_DISPATCH_K(pos.k, (k_cross_dense<KK><<<g, kBlock, 0, st>>>(c, v, elems, pos, m, mstride, mode, ws.partials,
                                                                  ws.counters, ro)));
  }
  MB_LAUNCHED();
  return MB_OK;
}

int launch_dm_trace(const double2* rho, int n, int nsamples, const Pos& pos, const double2* m, const ReduceWs& ws,
                    int slot, const ReduceOut& ro, cudaStream_t st) {
  if (nsamples <= 0) return MB_OK;
  dim3 g;
  int rc = reduce_grid((int64_t(1) << n) >> pos.k, nsamples, ws, slot, &g);
  if (rc) return rc;
  MB_DISPATCH_K(pos.k, (k_dm_trace<KK><<<g, kBlock, 0, st>>>(rho, n, pos, m, ws.partials, ws.counters, ro)));
  MB_LAUNCHED();
  return MB_OK;
}

int launch_dm_trace0(const double2* rho, int n, int nsamples, const double2* m, const ReduceWs& ws,
                     const ReduceOut& ro, cudaStream_t st) {
  if (nsamples <= 0) return MB_OK;
  dim3 g;
  int rc = reduce_grid(int64_t(1) << n, nsamples, ws, 0, &g);
  if (rc) return rc;
  k_dm_trace0<<<g, kBlock, 0, st>>>(rho, n, m, ws.partials, ws.counters, ro);
  MB_LAUNCHED();
  return MB_OK;
}

int launch_obs_apply(const double2* in, double2* out, int64_t elems, int nsamples, const Pos& pos, const double2* m,
                     int first, cudaStream_t st) {
  if (nsamples <= 0) return MB_OK;
  if (pos.k == 0) {
    k_obs_scalar<<<grid_for(elems * nsamples, kBlock), kBlock, 0, st>>>(in, out, elems * nsamples, m, first);
  } else {
    dim3 g = sample_grid(elems >> pos.k, nsamples);
    MB_DISPATCH_K(pos.k, (k_obs_apply<KK><<<g, kBlock, 0, st>>>(in, out, elems, pos, m, first)));
  }
  MB_LAUNCHED();
  return MB_OK;
}

int launch_marginal(const double2* v, int n, int is_dm, int nsamples, const int* qubits, int nq, double* out,
                    unsigned* flags, double tol, cudaStream_t st) {
  if (nsamples <= 0) return MB_OK;
  Readout ro{};
  ro.nq = nq;
  bool identity = nq == n;
  for (int j = 0; j < nq; ++j) {
    ro.q[j] = qubits[j];
    identity = identity && qubits[j] == j;
  }
  const int64_t dim = int64_t(1) << n;
  // A pure state is read whole and a density matrix only on its diagonal: 16 B per entry read.
  ProfScope ps(nq <= 12 && !identity ? "k_marginal_small" : "k_marginal_large", 16.0 * double(dim) * nsamples, st);
  if (nq <= 12 && !identity) {
    size_t shm = sizeof(double) << nq;
    k_marginal_small<<<sample_grid(dim, nsamples), kBlock, shm, st>>>(v, n, is_dm, ro, out, flags, tol);
  } else {
    k_marginal_large<<<sample_grid(dim, nsamples), kBlock, 0, st>>>(v, n, is_dm, ro, out, flags, tol, identity);
  }
  MB_LAUNCHED();
  return MB_OK;
}

int launch_bind(const BindRec* recs, int nrecs, const double* theta, int nslots, int rows, double2* table,
                int64_t stride, cudaStream_t st) {
  if (nrecs <= 0 || rows <= 0) return MB_OK;
  int64_t work = int64_t(nrecs) * rows;
  k_bind<<<grid_for(work, 128, int64_t(1) << 30), 128, 0, st>>>(recs, nrecs, theta, nslots, rows, table, stride);
  MB_LAUNCHED();
  return MB_OK;
}

}  // namespace mb
