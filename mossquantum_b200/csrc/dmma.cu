// K5: dense 4- and 5-qubit operators on the FP64 tensor cores (DMMA).
//
// The reference applies a 16x16 / 32x32 complex block to every group of amplitudes with
// scalar loops (_apply_fourbody_gate_impl!, _apply_fivebody_gate_impl!,
// src/backends/cpu/gates/threaded_long_range.jl:3-132). Here the amplitudes of GT = 64 groups
// form the columns of a complex D x GT matrix X (D = 2^k) and the block is one real GEMM
//   [Yr; Yi] = [[Ur, -Ui], [Ui, Ur]] [Xr; Xi]      (2D x 2D) x (2D x GT)
// issued as mma.sync m8n8k4 f64 tiles: each warp keeps the A fragments of its 8 output rows
// in registers for the whole launch and streams B fragments from shared memory.
// Staging: a tile's 2^k * 64 amplitudes are addressed through an index e whose bits map, in
// ascending order, onto the k target bits and the 6 lowest group bits, so a warp's 32
// consecutive e are 32 consecutive amplitudes (512 contiguous bytes) for any target set.
// Only the FP64 tensor pipe does arithmetic: 8 * 2^k flop per amplitude.
// Shared-memory layout of X (and Y): row r of 2D rows, column g of 64, at
// r * 68 + (g ^ ((r >> 2) & 7)). A half-warp's 64-bit accesses are conflict-free when their 16
// word addresses differ mod 16: the stride (4 mod 16 doubles) puts the four rows of a B
// fragment at offsets 0, 4, 8, 12 beside its four consecutive columns; the XOR, constant within
// each fragment's rows, keeps a staging access whose lanes hold 16 rows of one column distinct.
#include <algorithm>

#include "kernels.h"

namespace mb {
namespace {

constexpr int kGT = 64;           // groups per tile
constexpr int kDThreads = 256;    // 8 warps

struct DmmaArgs {
  int ebits;                      // k + 6
  int eaddr[11];                  // address bit of e-bit j (ascending)
  int etgt[11];                   // local target bit of e-bit j, or -1
  int egrp[11];                   // group-tile bit of e-bit j, or -1
  int gpos[64];                   // address bit of group bit i (non-target bits, ascending)
  int ngbits;                     // group bits per sample
  int64_t elems;                  // amplitudes per sample
  int64_t tiles_per_sample;
  int64_t ntiles;
};

__device__ __forceinline__ void dmma_m8n8k4(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

constexpr int kXS = kGT + 4;
__device__ __forceinline__ int xsw(int r, int g) { return r * kXS + (g ^ ((r >> 2) & 7)); }

template <int K>
__global__ void __launch_bounds__(kDThreads) k_dmma_block(double2* __restrict__ v, const DmmaArgs a,
                                                          const double2* __restrict__ m, int mode) {
  constexpr int D = 1 << K, M2 = 2 * D;
  constexpr int AS = M2 + 4;            // padded row strides (doubles): conflict-free fragments
  constexpr int MT = M2 / 8;            // 8-row output tiles
  constexpr int WPM = 8 / MT;           // warps per output tile
  constexpr int NT = (kGT / 8) / WPM;   // 8-column output tiles per warp
  constexpr int PER = D * kGT / kDThreads;
  extern __shared__ double smem[];
  double* As = smem;
  double* Xs = smem + M2 * AS;
  for (int e = threadIdx.x; e < D * D; e += kDThreads) {
    const int r = e % D, c = e / D;
    const double2 u = mat_at(m, D, r, c, mode);
    As[r * AS + c] = u.x;
    As[r * AS + D + c] = -u.y;
    As[(D + r) * AS + c] = u.y;
    As[(D + r) * AS + D + c] = u.x;
  }
  // Staging map of this thread's elements: e = threadIdx.x + i * 256 (bits of e are linear).
  int64_t t_addr = 0;
  int t_a = 0, t_g = 0;
  for (int j = 0; j < 8 && j < a.ebits; ++j)
    if ((threadIdx.x >> j) & 1) {
      t_addr |= int64_t(1) << a.eaddr[j];
      if (a.etgt[j] >= 0) t_a |= 1 << a.etgt[j];
      else t_g |= 1 << a.egrp[j];
    }
  int64_t i_addr[PER];
  int i_re[PER], i_im[PER];   // swizzled shared-memory slots of the element's real / imaginary part
#pragma unroll
  for (int i = 0; i < PER; ++i) {
    i_addr[i] = t_addr;
    int ia = t_a, ig = t_g;
    for (int j = 8; j < a.ebits; ++j)
      if ((i >> (j - 8)) & 1) {
        i_addr[i] |= int64_t(1) << a.eaddr[j];
        if (a.etgt[j] >= 0) ia |= 1 << a.etgt[j];
        else ig |= 1 << a.egrp[j];
      }
    i_re[i] = xsw(ia, ig);
    i_im[i] = xsw(D + ia, ig);
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int mt = warp % MT, nt0 = (warp / MT) * NT;
  double afr[M2 / 4];
#pragma unroll
  for (int ks = 0; ks < M2 / 4; ++ks) afr[ks] = As[(mt * 8 + (lane >> 2)) * AS + ks * 4 + (lane & 3)];

  for (int64_t tile = blockIdx.x; tile < a.ntiles; tile += gridDim.x) {
    const int64_t b = tile / a.tiles_per_sample;
    const int64_t tg = (tile - b * a.tiles_per_sample) * kGT;  // first group of the tile
    int64_t base = b * a.elems;
    for (int i = 6; i < a.ngbits; ++i)
      if ((tg >> i) & 1) base |= int64_t(1) << a.gpos[i];
    double2 x[PER];
#pragma unroll
    for (int i = 0; i < PER; ++i) x[i] = v[base | i_addr[i]];
#pragma unroll
    for (int i = 0; i < PER; ++i) {
      Xs[i_re[i]] = x[i].x;
      Xs[i_im[i]] = x[i].y;
    }
    __syncthreads();
    double acc[NT][2];
#pragma unroll
    for (int j = 0; j < NT; ++j) acc[j][0] = acc[j][1] = 0.0;
#pragma unroll
    for (int ks = 0; ks < M2 / 4; ++ks) {
      // rows ks*4 .. ks*4+3 share the swizzle (ks & 7)
      const double* xr = Xs + (ks * 4 + (lane & 3)) * kXS;
      const int c0 = nt0 * 8 + (lane >> 2);
#pragma unroll
      for (int j = 0; j < NT; ++j) dmma_m8n8k4(acc[j][0], acc[j][1], afr[ks], xr[(c0 + j * 8) ^ (ks & 7)]);
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < NT; ++j) {
      const int r = mt * 8 + (lane >> 2), c = (nt0 + j) * 8 + (lane & 3) * 2;
      Xs[xsw(r, c)] = acc[j][0];
      Xs[xsw(r, c + 1)] = acc[j][1];
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < PER; ++i) v[base | i_addr[i]] = make_double2(Xs[i_re[i]], Xs[i_im[i]]);
    __syncthreads();
  }
}

template <int K>
constexpr size_t dmma_smem() {
  return sizeof(double) * size_t(2 * (1 << K)) * size_t((2 * (1 << K) + 4) + kXS);
}

}  // namespace

// Dense k-qubit operator (k = 4 or 5, positions ascending) on every sample through the FP64
// tensor cores. Returns MB_EUNSUPPORTED when the shape does not fit (k outside 4..5, or
// fewer than 64 groups per sample), so callers can fall back to the plain kernel.
int launch_dmma(double2* v, int64_t elems, int nsamples, const Pos& pos, const double2* m, int mode,
                cudaStream_t st) {
  const int k = pos.k;
  if (k < 4 || k > 5) return MB_EUNSUPPORTED;
  int N = 0;
  while ((int64_t(1) << N) < elems) ++N;
  if ((int64_t(1) << N) != elems || N - k < 6 || N > 62) return MB_EUNSUPPORTED;
  for (int j = 0; j < k; ++j)
    if (pos.p[j] < 0 || pos.p[j] >= N || (j && pos.p[j] <= pos.p[j - 1])) return MB_EUNSUPPORTED;
  DmmaArgs a{};
  a.ngbits = N - k;
  int gi = 0;
  for (int q = 0, t = 0; q < N; ++q) {
    if (t < k && pos.p[t] == q) {
      ++t;
      continue;
    }
    a.gpos[gi++] = q;
  }
  // e-bits: the k targets and the 6 lowest group bits, in ascending address order.
  a.ebits = k + 6;
  int j = 0;
  for (int q = 0, t = 0, g = 0; q < N && j < a.ebits; ++q) {
    if (t < k && pos.p[t] == q) {
      a.eaddr[j] = q;
      a.etgt[j] = t++;
      a.egrp[j] = -1;
      ++j;
    } else if (g < 6) {
      a.eaddr[j] = q;
      a.etgt[j] = -1;
      a.egrp[j] = g++;
      ++j;
    } else if (t >= k) {
      break;
    } else {
      ++g;  // a group bit above the tile: covered by the tile base
    }
  }
  if (j != a.ebits) return MB_EUNSUPPORTED;
  a.elems = elems;
  a.tiles_per_sample = (int64_t(1) << a.ngbits) / kGT;
  a.ntiles = a.tiles_per_sample * nsamples;
  if (a.ntiles == 0) return MB_OK;
  size_t shm = 0;
  int per_sm = 1;
  if (k == 4) {
    shm = dmma_smem<4>();
    cudaFuncSetAttribute(k_dmma_block<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(shm));
  } else {
    shm = dmma_smem<5>();
    cudaFuncSetAttribute(k_dmma_block<5>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(shm));
  }
  per_sm = std::max(1, int((227 * 1024) / (shm + 1024)));
  const int64_t grid = std::min<int64_t>(a.ntiles, int64_t(148) * std::min(per_sm, 4));
  {
    ProfScope ps(k == 4 ? "k_dmma_block4" : "k_dmma_block5", 32.0 * double(elems) * nsamples, st,
                 8.0 * double(1 << k) * double(elems) * nsamples);
    if (k == 4) k_dmma_block<4><<<unsigned(grid), kDThreads, shm, st>>>(v, a, m, mode);
    else k_dmma_block<5><<<unsigned(grid), kDThreads, shm, st>>>(v, a, m, mode);
  }
  MB_LAUNCHED();
  return MB_OK;
}

}  // namespace mb
