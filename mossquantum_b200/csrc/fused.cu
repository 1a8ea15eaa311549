// Fused-pass execution: gate-stream scheduler (host) and the K1/K2 pass kernels.
//
// The reference applies every gate as one full sweep over the state (threaded_short_range.jl,
// threaded_long_range.jl). Here the compiled circuit is cut into passes; one pass reads and
// writes the state once and applies every gate it holds:
//   PASS_TILE (K1)  a tile of 2^t amplitudes (t = 10..12) over the bit set {0,1,2} ∪ H (H a
//                   window of higher bits) or the low bits {0..t-1}, staged into shared memory
//                   by TMA (cp.async.bulk.tensor, 128-byte swizzle) and processed in
//                   register stages of 2^R amplitudes per thread;
//   PASS_REG  (K2)  a coalesced strided sweep: each thread holds 2^R amplitudes 2^h apart
//                   (R high bits), warps cover 32 consecutive low indices (512 B per load);
//   PASS_PLAIN      one plain kernel for an instruction the register stages cannot hold
//                   (dense gates on 3..5 qubits, 2-qubit channels).
// Gates are taken into a pass greedily in circuit order; a gate may move ahead of skipped
// gates only when it commutes with all of them (disjoint non-diagonal supports), so the
// result equals the sequential product. Density matrices run as 2n-bit vectors: U on the
// row bits and conj(U) on the column bits, channels as supermatrices.
#include <cuda.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <functional>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <unordered_map>

#include "fused_kernels.cuh"
#include "family.cuh"
#include "fusemat.cuh"
#include "jit.h"

namespace mb {

namespace {

typedef std::complex<double> cd;

// ---------------------------------------------------------------------------------------------
// Kernels
// ---------------------------------------------------------------------------------------------
template <int R> struct TileBounds;
template <> struct TileBounds<4> { static constexpr int threads = 256, blocks = 1; };
template <> struct TileBounds<5> { static constexpr int threads = 128, blocks = 1; };

template <int R, bool U2>
__global__ void __launch_bounds__(TileBounds<R>::threads, TileBounds<R>::blocks)
    k_tile_pass(const __grid_constant__ CUtensorMap tmap, const TileArgs a) {
  // Two tile buffers: while the CTA works on tile i in one buffer, TMA stores tile i-1 and
  // loads tile i+1 through the other.
  extern __shared__ unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ int s_abort;
  double2* buf0 = reinterpret_cast<double2*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  double2* bufs[2] = {buf0, buf0 + (size_t(1) << a.t)};
  const uint32_t tile_bytes = 16u << a.t;
  if (threadIdx.x == 0) {
    fk::mbar_init(&bar[0], 1);
    fk::mbar_init(&bar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    s_abort = 0;
  }
  __syncthreads();
  // Tile geometry: global base index (zeros at the tile bits) and TMA coordinates.
  auto geometry = [&](int64_t tile, int* c, uint64_t* gbase, int* sample) {
    const int b = int(tile / a.tiles_per_sample);
    uint64_t base = uint64_t(tile - int64_t(b) * a.tiles_per_sample);
    for (int q = 0; q < a.t; ++q) {
      const int p = a.bits[q];
      const uint64_t low = base & ((uint64_t(1) << p) - 1);
      base = ((base >> p) << (p + 1)) | low;
    }
    for (int d = 0; d < a.ndims; ++d) {
      if (a.start[d] < 0) c[d] = b;
      else if (d == 0) c[d] = int(2 * (base & ((uint64_t(1) << a.extb[0]) - 1)));
      else c[d] = int((base >> a.start[d]) & ((uint64_t(1) << a.extb[d]) - 1));
    }
    *gbase = base;
    *sample = b;
  };
  uint32_t phase[2] = {0u, 0u};
  int64_t tile = blockIdx.x;
  if (threadIdx.x == 0 && tile < a.ntiles) {
    int c[5];
    uint64_t gb;
    int b;
    geometry(tile, c, &gb, &b);
    fk::mbar_expect_tx(&bar[0], tile_bytes);
    fk::tma_load(&tmap, bufs[0], &bar[0], a.ndims, c);
  }
  for (int it = 0; tile < a.ntiles; ++it, tile += gridDim.x) {
    const int cur = it & 1;
    const int64_t next = tile + gridDim.x;
    if (threadIdx.x == 0 && next < a.ntiles) {
      int c[5];
      uint64_t gb;
      int b;
      geometry(next, c, &gb, &b);
      fk::bulk_wait_read();  // the store that last used the other buffer has read it
      fk::mbar_expect_tx(&bar[cur ^ 1], tile_bytes);
      fk::tma_load(&tmap, bufs[cur ^ 1], &bar[cur ^ 1], a.ndims, c);
    }
    int c[5];
    uint64_t base;
    int b;
    geometry(tile, c, &base, &b);
    double2* tl = bufs[cur];
    if (!fk::mbar_wait(&bar[cur], phase[cur])) {
      atomicOr(a.err, 1u);
      s_abort = 1;
    }
    phase[cur] ^= 1u;
    __syncthreads();
    if (s_abort) break;
    for (int s = 0; s < a.nstages; ++s) {
      const StageDesc& sd = a.stages[s];
      int reg[kMaxRegBits];
#pragma unroll
      for (int k = 0; k < R; ++k) reg[k] = sd.reg[k];
      uint32_t lbase = 0;
      for (int q = 0; q < sd.ntid; ++q) lbase |= ((threadIdx.x >> q) & 1u) << sd.tid[q];
      double2 v[1 << R];
#pragma unroll
      for (int j = 0; j < (1 << R); ++j) v[j] = tl[fk::swz(lbase | uint32_t(fk::reg_offset<R>(j, reg)))];
      fk::run_mops<R, U2>(v, a.mops + sd.op0, sd.nops, lbase, reg, base, a.table, a.xtab, a.xtabs + b * a.xrow,
                          a.tstride, b);
#pragma unroll
      for (int j = 0; j < (1 << R); ++j) tl[fk::swz(lbase | uint32_t(fk::reg_offset<R>(j, reg)))] = v[j];
      __syncthreads();
    }
    fk::fence_async_smem();
    __syncthreads();
    if (threadIdx.x == 0) fk::tma_store(&tmap, tl, a.ndims, c);
  }
  if (threadIdx.x == 0) fk::bulk_wait_all();
}

template <int R, bool U2>
__global__ void __launch_bounds__(128) k_reg_pass(double2* __restrict__ v, const RegArgs a) {
  int reg[kMaxRegBits];
#pragma unroll
  for (int k = 0; k < R; ++k) reg[k] = a.reg[k];
  const int64_t total = a.groups * a.nsamples;
  for (int64_t g = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; g < total; g += int64_t(gridDim.x) * blockDim.x) {
    const int b = int(g / a.groups);
    uint64_t base = uint64_t(g - int64_t(b) * a.groups);
#pragma unroll
    for (int k = 0; k < R; ++k) {
      const int p = reg[k];
      const uint64_t low = base & ((uint64_t(1) << p) - 1);
      base = ((base >> p) << (p + 1)) | low;
    }
    double2* vs = v + (int64_t(b) << a.N);
    double2 x[1 << R];
#pragma unroll
    for (int j = 0; j < (1 << R); ++j) x[j] = vs[base | fk::reg_offset<R>(j, reg)];
    fk::run_mops<R, U2>(x, a.mops, a.nops, base, reg, 0, a.table, a.xtab, a.xtabs + b * a.xrow, a.tstride, b);
#pragma unroll
    for (int j = 0; j < (1 << R); ++j) vs[base | fk::reg_offset<R>(j, reg)] = x[j];
  }
}

// Per-sample products of the fused single-qubit runs (after binding): row b of the derived
// table's per-sample region gets every record's product formed from table row b.
__global__ void k_fuse(const FuseRec* __restrict__ recs, int nrecs, const FuseComp* __restrict__ comps,
                       const double2* __restrict__ table, int64_t tstride, double2* __restrict__ xs, int64_t xrow,
                       int rows) {
  const int64_t idx = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (idx >= int64_t(nrecs) * rows) return;
  const int b = int(idx / nrecs);
  const FuseRec r = recs[idx % nrecs];
  double2 M[16];
  fuse_product(r, comps, table, table + int64_t(b) * tstride, M);
  double2* out = xs + int64_t(b) * xrow + r.out;
  for (int e = 0; e < r.d * r.d; ++e) out[e] = M[e];
}

// ---------------------------------------------------------------------------------------------
// Host: fused ops
// ---------------------------------------------------------------------------------------------
// Persistent uneven batch: one launch over samples of different register sizes, each with its
// own parameters. The work items are (sample, pass, chunk of up to 2^15 amplitudes' tiles),
// ordered by pass index first, so every pass-0 chunk of every sample comes before any pass-1
// chunk; CTAs take items from a work counter. Before an item of pass p a CTA waits until its
// sample has completed every chunk of pass p-1 (a per-sample counter); those chunks were all
// taken earlier by running CTAs, so the wait always ends (it is also bounded, and sets the
// error flag). Pass 0 generates |0..0> instead of loading. Chunks of one pass touch disjoint
// amplitudes; the state is read through L2 (ld.global.cg), so another SM's writes of the
// previous pass are seen after the counter. Two launches before it bind every sample's
// parameter row and form its fused single-qubit products, for all sizes at once (the pass
// kernel reads the tables through the read-only cache, so they are written before it starts).
constexpr int kUnevenThreads = 128;
constexpr int kUnevenMaxTile = 11;   // 2^11-amplitude tiles, 16 amplitudes per thread
constexpr int kUnevenJitTile = 10;   // specialised form (mbk_uneven): 2^10 tiles, 8 per thread

struct UnevenGroup {
  int n;                      // amplitude bits of one sample
  int B;                      // samples
  int pass0, npasses;         // this size's passes in the plan's pass array
  int sample0;                // first of this group's per-sample completion counters
  int nchunks;                // items per pass and sample
  int64_t bind0, fuse0;       // first work item of this group in the bind and fuse launches
  int nbinds, nslots;
  const BindRec* binds;
  const double* theta;        // nslots values per sample
  int nrecs;
  const FuseRec* recs;
  const FuseComp* comps;
  double2* states;            // samples back to back
  double2* table;             // matrix table, one row of tstride entries per sample
  int64_t tstride;
  const double2* xtab;        // derived coefficients, then per-sample rows of xrow entries
  double2* xtabs;
  int64_t xrow;
};

struct UnevenPass {
  int t, nstages;
  int bits[16];
  const StageDesc* stages;
  const MOp* mops;
};

// Group of work item w (groups ordered by their first item).
__device__ __forceinline__ int uneven_group_of(const UnevenGroup* g, int ng, int64_t w, bool fuse) {
  int i = 0;
  while (i + 1 < ng && (fuse ? g[i + 1].fuse0 : g[i + 1].bind0) <= w) ++i;
  return i;
}

// Parameter binding of every sample of every group: item = (group, sample, bind record).
__global__ void k_uneven_bind(const UnevenGroup* __restrict__ groups, int ng, int64_t total) {
  const int64_t w = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (w >= total) return;
  const UnevenGroup& G = groups[uneven_group_of(groups, ng, w, false)];
  const int64_t r = w - G.bind0;
  const int b = int(r / G.nbinds), q = int(r % G.nbinds);
  const BindRec rc = G.binds[q];
  const double th = rc.slot >= 0 ? G.theta[int64_t(b) * G.nslots + rc.slot] : rc.value;
  bind_record(rc, th, G.table, G.table + int64_t(b) * G.tstride);
}

// Fused single-qubit products of every sample of every group: item = (group, sample, record).
__global__ void k_uneven_fuse(const UnevenGroup* __restrict__ groups, int ng, int64_t total) {
  const int64_t w = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (w >= total) return;
  const UnevenGroup& G = groups[uneven_group_of(groups, ng, w, true)];
  const int64_t r = w - G.fuse0;
  const int b = int(r / G.nrecs), q = int(r % G.nrecs);
  const FuseRec rec = G.recs[q];
  double2 M[16];
  fuse_product(rec, G.comps, G.table, G.table + int64_t(b) * G.tstride, M);
  double2* out = G.xtabs + int64_t(b) * G.xrow + rec.out;
  for (int e = 0; e < rec.d * rec.d; ++e) out[e] = M[e];
}

// Work item: x = group, y = sample, z = pass index within the group, w = chunk.
template <bool U2>
__global__ void __launch_bounds__(kUnevenThreads, 2)
    k_uneven(const UnevenGroup* __restrict__ groups, const UnevenPass* __restrict__ passes,
             const int4* __restrict__ items, int nitems, unsigned* next, unsigned* done, int zero_init,
             unsigned* err) {
  constexpr int R = 4;
  extern __shared__ unsigned char smem_raw[];
  double2* tl = reinterpret_cast<double2*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* loc = reinterpret_cast<uint64_t*>(tl + (1 << kUnevenMaxTile));
  __shared__ int s_item, s_ok;
  const int tx = threadIdx.x;
  for (;;) {
    if (tx == 0) s_item = int(atomicAdd(next, 1u));
    __syncthreads();
    const int item = s_item;
    if (item >= nitems) break;
    const int4 it = items[item];
    const UnevenGroup& G = groups[it.x];
    const int b = it.y, pi = it.z, chunk = it.w;
    unsigned* cnt = done + G.sample0 + b;
    if (tx == 0) {
      // every chunk of the previous passes of this sample
      const unsigned need = unsigned(pi) * unsigned(G.nchunks);
      int ok = 1;
      for (uint32_t spin = 0; atomicAdd(cnt, 0u) < need; ++spin) {
        if (spin > (1u << 24)) {
          atomicOr(err, 1u);
          ok = 0;
          break;
        }
        __nanosleep(64);
      }
      __threadfence();
      s_ok = ok;
    }
    __syncthreads();
    if (!s_ok) break;
    const UnevenPass& P = passes[G.pass0 + pi];
    const int t = P.t, T = 1 << t;
    const int64_t dim = int64_t(1) << G.n;
    double2* v = G.states + int64_t(b) * dim;
    const double2* xs = G.xtabs ? G.xtabs + int64_t(b) * G.xrow : nullptr;
    for (int l = tx; l < T; l += kUnevenThreads) {
      uint64_t o = 0;
      for (int q = 0; q < t; ++q) o |= uint64_t((l >> q) & 1) << P.bits[q];
      loc[l] = o;
    }
    __syncthreads();
    const int64_t ntiles = dim >> t;
    const int64_t per = (ntiles + G.nchunks - 1) / G.nchunks;
    const int64_t t0 = int64_t(chunk) * per, t1 = t0 + per < ntiles ? t0 + per : ntiles;
    const bool gen = zero_init && pi == 0;
    for (int64_t tile = t0; tile < t1; ++tile) {
      uint64_t base = uint64_t(tile);
      for (int q = 0; q < t; ++q) {
        const int p = P.bits[q];
        base = ((base >> p) << (p + 1)) | (base & ((uint64_t(1) << p) - 1));
      }
      for (int l = tx; l < T; l += kUnevenThreads)
        tl[fk::swz(uint32_t(l))] = gen ? make_double2((base | loc[l]) == 0 ? 1.0 : 0.0, 0.0) : __ldcg(v + (base | loc[l]));
      __syncthreads();
      for (int s = 0; s < P.nstages; ++s) {
        const StageDesc& sd = P.stages[s];
        int reg[kMaxRegBits];
#pragma unroll
        for (int k = 0; k < R; ++k) reg[k] = sd.reg[k];
        const int vthreads = 1 << sd.ntid;
        for (int vt = tx; vt < vthreads; vt += kUnevenThreads) {
          uint32_t lbase = 0;
          for (int q = 0; q < sd.ntid; ++q) lbase |= ((uint32_t(vt) >> q) & 1u) << sd.tid[q];
          double2 a[1 << R];
#pragma unroll
          for (int j = 0; j < (1 << R); ++j) a[j] = tl[fk::swz(lbase | uint32_t(fk::reg_offset<R>(j, reg)))];
          fk::run_mops<R, U2>(a, P.mops + sd.op0, sd.nops, lbase, reg, base, G.table, G.xtab, xs, G.tstride, b);
#pragma unroll
          for (int j = 0; j < (1 << R); ++j) tl[fk::swz(lbase | uint32_t(fk::reg_offset<R>(j, reg)))] = a[j];
        }
        __syncthreads();
      }
      for (int l = tx; l < T; l += kUnevenThreads) v[base | loc[l]] = tl[fk::swz(uint32_t(l))];
      __syncthreads();
    }
    // publish this chunk: every thread's stores, then the counter
    __threadfence();
    __syncthreads();
    if (tx == 0) atomicAdd(cnt, 1u);
  }
}

// ---------------------------------------------------------------------------------------------
enum { F_UNFUSABLE = -1 };

}  // namespace

struct FOp {
  int type = F_UNFUSABLE;     // MopType or F_UNFUSABLE
  int nb = 0;                 // bits of the (ordered) local matrix
  int bits[10] = {0};         // global bit of local bit j
  uint64_t all = 0, nd = 0;   // all bits / non-diagonal (target) bits
  int tgt[2] = {0, 0};
  int ntgt = 0;
  int ctrl[4] = {0};
  int nctrl = 0;
  int off[16] = {0};
  uint32_t active = 0;
  int conj = 0, param = 0;
  bool neg = false;           // MOP_CPHASE with factor -1 (a sign flip)
  int slot = -1;              // MOP_GRAD / MOP_GRADP: parameter slot
  int pauli = 0;              // MOP_GRADP: generator code (1 X, 2 Y, 3 Z, 4 PHASE)
  int only = 0;               // reverse sweeps: 0 both states, 1 y only, 2 delta only
  // plain fallback
  int cls = CLS_DENSE;
  int mat_off = 0, mode = MAT_PLAIN;
  uint32_t pactive = 0;
  int sigma[32];
  int d = 1;
  // Phase bookkeeping of the forward schedules (merge_phases): a fixed single-qubit phase
  // diag(1, ph) on bits[0] that may be merged with its neighbours, and a global factor.
  bool merge = false;
  cd ph = cd(1, 0), glob = cd(1, 0);
};

struct Schedule {
  std::vector<double2> xtab;      // derived coefficients (kXtabFlag offsets), the same for every sample
  double2* d_xtab = nullptr;      // xtab, then nsamples rows of xrow per-sample entries
  int xrow = 0;                   // per-sample entries (fused products) per row
  bool fuse = true;               // bind-time fusion of single-qubit runs
  std::vector<FuseComp> fcomps;   // per-sample fusion records, formed by k_fuse after binding
  std::vector<FuseRec> frecs;
  FuseComp* d_fcomps = nullptr;
  FuseRec* d_frecs = nullptr;
  int N = 0, dm = 0, t = 0, R = 0, nsamples = 1;
  int lo = 0, hi = -1;  // instruction range [lo, hi) of the circuit
  int adjoint = 0;      // reverse sweep with gradient accumulators
  int* d_gslots = nullptr;
  int max_grad = 0;     // most gradient accumulators in one pass
  int jit = 0;  // 0 not tried, 1 specialised kernels ready, -1 interpreter kernels
  bool dagger = false;
  bool unschedulable = false;  // an adjoint op that no pass can hold
  bool tile_only = false;      // built without register passes
  std::vector<FOp> fops;
  std::vector<Pass> passes;
  StageDesc* d_stages = nullptr;
  MOp* d_mops = nullptr;
};

namespace {

// Algorithmic FP64 flops per amplitude of one micro-op: 8*2^k for a dense k-qubit complex
// gate (2^k complex multiply-adds), scaled by the fraction of amplitudes a controlled or
// diagonal op touches; 8 for a 2x2 with real (or real-diagonal, imaginary-off-diagonal)
// entries, 6 for a rotation applied as three shears; swaps and sign flips count zero.
static double mop_flops(const MOp& m) {
  switch (m.type) {
    case MOP_U1: return 16.0;
    case MOP_CTRL: return 16.0 / double(1 << m.nsel);
    case MOP_U2: return 32.0;
    case MOP_DIAG: return 6.0 * __builtin_popcount(m.active) / double(1 << m.nsel);
    case MOP_CPHASE: return m.r1 ? 0.0 : 6.0 / double(1 << m.nsel);
    case MOP_GRAD: return 8.0 * double(1 << m.nsel) + 8.0;
    case MOP_RROT: case MOP_IROT: return 8.0;  // four real multiply-adds per amplitude
    case MOP_LIFT: return 6.0;                 // three fused multiply-adds per amplitude
    case MOP_GRADP: return 4.0;                // two multiply-adds per amplitude
    case MOP_CHAN: return 4.0;                 // 12 real multiply-adds per 4 amplitudes
    default: return 0.0;
  }
}

static double pass_flops_per_amp(const Pass& p, bool dual) {
  double f = 0;
  for (const MOp& m : p.mops)
    f += (dual && m.type != MOP_GRAD && m.type != MOP_GRADP) ? 2.0 * mop_flops(m) : mop_flops(m);
  return f;
}

static bool is_one(double2 x) { return x.x == 1.0 && x.y == 0.0; }
static bool is_zero(double2 x) { return x.x == 0.0 && x.y == 0.0; }

// Controlled single-target structure of a fixed ordered matrix: identity unless every
// bit other than `tj` is 1. Returns the target local bit or -1.
static int controlled_target(const double2* M, int k) {
  const int d = 1 << k;
  for (int tj = 0; tj < k; ++tj) {
    const int tb = 1 << tj, cm = (d - 1) & ~tb;
    bool ok = true;
    for (int r = 0; r < d && ok; ++r)
      for (int c = 0; c < d && ok; ++c) {
        const double2 x = M[r + c * d];
        if ((r & ~tb) != (c & ~tb)) ok = is_zero(x);
        else if ((r & cm) != cm) ok = (r == c) ? is_one(x) : is_zero(x);
      }
    if (ok) return tj;
  }
  return -1;
}

static void finalize_masks(FOp& f) {
  f.all = 0;
  for (int j = 0; j < f.nb; ++j) f.all |= uint64_t(1) << f.bits[j];
  f.nd = 0;
  for (int j = 0; j < f.ntgt; ++j) f.nd |= uint64_t(1) << f.tgt[j];
}

// Fused op of one gate half (row bits or, with conj, column bits of a density matrix).
static FOp gate_fop(mb_circuit c, const COp& op, int shift, int conj, bool dagger) {
  FOp f;
  f.nb = op.k;
  for (int j = 0; j < op.k; ++j) f.bits[j] = op.pos[j] + shift;
  f.conj = conj;
  f.param = op.parametric ? 1 : 0;
  f.mat_off = op.mat_off;
  f.d = 1 << op.k;
  f.cls = op.cls;
  f.pactive = op.active;
  std::memcpy(f.sigma, dagger ? op.sigma_inv : op.sigma, sizeof(f.sigma));
  f.mode = dagger ? (conj ? MAT_TRANSPOSE : MAT_ADJOINT) : (conj ? MAT_CONJ : MAT_PLAIN);
  const int d = f.d;
  // Element (r, c) of the effective matrix (U, conj U, U' or U^T) as a table offset; the
  // conj flag is toggled for the adjoint.
  auto off = [&](int r, int cc) { return dagger ? op.mat_off + cc + r * d : op.mat_off + r + cc * d; };
  const int fconj = dagger ? !conj : conj;
  if (op.k == 0) return f;  // global scalar: plain path
  if (op.cls == CLS_DIAG) {
    const int nact = __builtin_popcount(op.active);
    if (nact == 1 && op.active == (1u << (d - 1)) && op.k <= 4) {
      // Phase on the all-ones entry: CZ, CPHASE, CCPHASE, PHASE, Z, S, T.
      f.type = MOP_CPHASE;
      f.off[0] = off(d - 1, d - 1);
      for (int j = 0; j < op.k; ++j) f.ctrl[f.nctrl++] = f.bits[j];
      if (!op.parametric) {
        const double2 x = c->fixed_table[op.mat_off + (d - 1) * (d + 1)];
        f.neg = x.x == -1.0 && x.y == 0.0;
      }
      f.conj = fconj;
      finalize_masks(f);
      return f;
    }
    if (op.k <= 3) {
      // One complex multiply per touched amplitude, no register target needed (RZ, CRZ, ...).
      f.type = MOP_DIAG;
      for (int a = 0; a < d; ++a) f.off[a] = off(a, a);
      f.active = op.active;
      f.conj = fconj;
      finalize_masks(f);
      return f;
    }
    // Larger diagonals that are identity unless all bits but one are set: controlled 2x2.
    for (int tj = 0; tj < op.k && op.k >= 1; ++tj) {
      const int tb = 1 << tj, cm = (d - 1) & ~tb;
      uint32_t ctl = 0;
      for (int a = 0; a < d; ++a)
        if ((a & cm) == cm) ctl |= 1u << a;
      if ((op.active & ~ctl) == 0) {
        f.tgt[0] = f.bits[tj];
        f.ntgt = 1;
        for (int j = 0; j < op.k; ++j)
          if (j != tj) f.ctrl[f.nctrl++] = f.bits[j];
        f.off[0] = off(cm, cm);
        f.off[1] = off(cm | tb, cm);
        f.off[2] = off(cm, cm | tb);
        f.off[3] = off(cm | tb, cm | tb);
        f.type = f.nctrl ? MOP_CTRL : MOP_U1;
        if (f.nctrl > 4) f.type = F_UNFUSABLE;
        f.conj = fconj;
        finalize_masks(f);  // the target must sit in a register like any 2x2 op
        return f;
      }
    }
    if (op.k > 3) return f;
    f.type = MOP_DIAG;
    for (int a = 0; a < d; ++a) f.off[a] = off(a, a);
    f.active = op.active;
    f.conj = fconj;
    finalize_masks(f);
    return f;
  }
  int tj = -1;
  bool is_x = false;
  if (op.parametric) {
    if (op.family == MB_FAM_CRX || op.family == MB_FAM_CRY) {
      for (int j = 0; j < op.k; ++j) {
        // the target is the bit that carries own-order bit 1 (second position)
        const BindRec* br = nullptr;
        for (auto& r : c->binds)
          if (r.mat_off == op.mat_off) br = &r;
        if (br && br->perm[1 << j] == 2) tj = j;
      }
    }
  } else if (op.k >= 2) {
    tj = controlled_target(c->fixed_table.data() + op.mat_off, op.k);
  }
  if (op.k == 1) tj = 0;
  if (tj >= 0) {
    const int tb = 1 << tj, cm = (d - 1) & ~tb;
    f.tgt[0] = f.bits[tj];
    f.ntgt = 1;
    for (int j = 0; j < op.k; ++j)
      if (j != tj) f.ctrl[f.nctrl++] = f.bits[j];
    f.off[0] = off(cm, cm);
    f.off[1] = off(cm | tb, cm);
    f.off[2] = off(cm, cm | tb);
    f.off[3] = off(cm | tb, cm | tb);
    if (!op.parametric) {
      const double2* M = c->fixed_table.data();
      is_x = is_zero(M[f.off[0]]) && is_one(M[f.off[1]]) && is_one(M[f.off[2]]) && is_zero(M[f.off[3]]);
    }
    f.type = is_x ? MOP_CTRLX : (f.nctrl ? MOP_CTRL : MOP_U1);
    if (f.type == MOP_U1) {
      // Real (RY, H) and real-diagonal / imaginary-off-diagonal (RX) matrices take half the
      // arithmetic of a complex 2x2; the structure holds for U, conj U, U' and U^T alike.
      if (op.parametric) {
        if (op.family == MB_FAM_RY) f.type = MOP_RROT;
        else if (op.family == MB_FAM_RX) f.type = MOP_IROT;
      } else {
        const double2* M = c->fixed_table.data();
        const double2 e00 = M[f.off[0]], e10 = M[f.off[1]], e01 = M[f.off[2]], e11 = M[f.off[3]];
        if (e00.y == 0.0 && e10.y == 0.0 && e01.y == 0.0 && e11.y == 0.0) f.type = MOP_RROT;
        else if (e00.y == 0.0 && e11.y == 0.0 && e01.x == 0.0 && e10.x == 0.0) f.type = MOP_IROT;
      }
    }
    if (f.nctrl > 4) f.type = F_UNFUSABLE;
    f.conj = fconj;
    finalize_masks(f);
    return f;
  }
  if (op.k == 2) {
    f.type = MOP_U2;
    for (int r = 0; r < 4; ++r)
      for (int cc = 0; cc < 4; ++cc) f.off[r + 4 * cc] = off(r, cc);
    f.tgt[0] = f.bits[0];
    f.tgt[1] = f.bits[1];
    f.ntgt = 2;
    f.conj = fconj;
    finalize_masks(f);
  }
  return f;
}

// Unfusable ops act densely on all their bits.
static void mark_unfusable_masks(FOp& f) {
  if (f.type != F_UNFUSABLE) return;
  f.all = 0;
  for (int j = 0; j < f.nb; ++j) f.all |= uint64_t(1) << f.bits[j];
  f.nd = f.all;
}

// A fixed 2x2 as E = g * diag(1, A) * R * diag(1, B), R = [[c, -s], [s, c]] with c = |e00| and
// s = |e10|, so that R runs as three shears with t = s / (1 + c) <= 1. Returns false (the gate
// stays a complex 2x2) unless E is unitary to 1e-14 and the factors, with R as the product of
// its shears, reproduce E to 1e-14.
static bool decompose_u2(const cd E[4], cd* g, cd* A, cd* B, double* mt, double* sn) {
  const cd u00 = std::conj(E[0]) * E[0] + std::conj(E[1]) * E[1];
  const cd u01 = std::conj(E[0]) * E[2] + std::conj(E[1]) * E[3];
  const cd u11 = std::conj(E[2]) * E[2] + std::conj(E[3]) * E[3];
  if (std::abs(u00 - 1.0) > 1e-14 || std::abs(u11 - 1.0) > 1e-14 || std::abs(u01) > 1e-14) return false;
  const double c = std::abs(E[0]), s = std::abs(E[1]);
  if (!(s > 0.0)) return false;
  *g = c > 0.0 ? E[0] / c : cd(1, 0);
  *A = E[1] / (*g * s);
  *B = -E[2] / (*g * s);
  const double t = s / (1.0 + c);
  const double r00 = 1.0 - t * s, r01 = -2.0 * t + s * t * t, r10 = s, r11 = 1.0 - s * t;
  const cd F[4] = {*g * r00, *g * *A * r10, *g * r01 * *B, *g * *A * r11 * *B};
  for (int e = 0; e < 4; ++e)
    if (std::abs(F[e] - E[e]) > 1e-14) return false;
  *mt = -t;
  *sn = s;
  return true;
}

static int xtab_push(std::vector<double2>* xt, double2 v) {
  xt->push_back(v);
  return int(xt->size() - 1) | kXtabFlag;
}

// diag(1, ph) on global bit `bit` as a single-selector phase micro-op (a sign flip for -1).
static FOp phase_fop(int bit, cd ph, std::vector<double2>* xt) {
  FOp f;
  f.type = MOP_CPHASE;
  f.nb = 1;
  f.bits[0] = bit;
  f.ctrl[0] = bit;
  f.nctrl = 1;
  f.cls = CLS_DIAG;
  f.neg = ph == cd(-1, 0);
  f.off[0] = xtab_push(xt, make_double2(ph.real(), ph.imag()));
  finalize_masks(f);
  return f;
}

// Phase merging for forward schedules. Every fixed single-qubit phase is held back and
// multiplied into the next phase on the same bit until a non-diagonal op acts on that bit
// (all diagonal ops commute, and a phase on a control bit commutes with the controlled op),
// so a chain U3, CZ, U3 on one qubit costs one phase between the two rotations. Global
// factors are collected into one diagonal micro-op (pure states; for density matrices the row
// and column factors cancel).
static void merge_phases(std::vector<FOp>& seq, bool dm, std::vector<double2>* xt) {
  std::vector<FOp> out;
  out.reserve(seq.size());
  cd pend[64];
  bool has[64] = {false};
  cd glob(1, 0);
  auto flush = [&](int q) {
    if (!has[q]) return;
    has[q] = false;
    if (pend[q] != cd(1, 0)) out.push_back(phase_fop(q, pend[q], xt));
  };
  for (FOp& f : seq) {
    if (f.merge) {
      const int q = f.bits[0];
      pend[q] = has[q] ? pend[q] * f.ph : f.ph;
      has[q] = true;
      glob *= f.glob;
      continue;
    }
    for (uint64_t m = f.nd; m; m &= m - 1) flush(__builtin_ctzll(m));
    out.push_back(std::move(f));
  }
  for (int q = 0; q < 64; ++q) flush(q);
  if (!dm && glob != cd(1, 0)) {
    FOp f;
    f.type = MOP_DIAG;
    f.nb = 1;
    f.bits[0] = 0;
    f.cls = CLS_DIAG;
    f.off[0] = f.off[1] = xtab_push(xt, make_double2(glob.real(), glob.imag()));
    f.active = 3;
    finalize_masks(f);
    out.push_back(f);
  }
  seq.swap(out);
}

// A fixed single-qubit op of a forward schedule (a gate half, or a fused run formed on the host):
// a general unitary becomes phase, three-shear rotation, phase (and a global factor); a diagonal
// becomes a phase and a global factor. The phases are marked for merge_phases. Returns false to
// keep `f` as it is.
static bool split_fixed_1q(mb_circuit c, const FOp& f, bool dm, std::vector<double2>* xt, std::vector<FOp>& seq) {
  if (f.param || f.type == F_UNFUSABLE) return false;
  auto eff = [&](int e) {
    const int off = f.off[e];
    const double2 x = (off & kXtabFlag) ? (*xt)[off & ~kXtabFlag] : c->fixed_table[off];
    return cd(x.x, f.conj ? -x.y : x.y);
  };
  const int q = f.bits[0];
  if (f.type == MOP_DIAG && f.nb == 1) {
    const cd d0 = (f.active & 1) ? eff(0) : cd(1, 0), d1 = (f.active & 2) ? eff(1) : cd(1, 0);
    if (!(std::abs(d0) > 0.0)) return false;
    if (dm && (std::abs(std::abs(d0) - 1.0) > 1e-14 || std::abs(std::abs(d1) - 1.0) > 1e-14)) return false;
    FOp p;
    p.merge = true;
    p.bits[0] = q;
    p.ph = d1 / d0;
    p.glob = d0;
    seq.push_back(p);
    return true;
  }
  if (f.type == MOP_CPHASE && f.nctrl == 1) {
    FOp p;
    p.merge = true;
    p.bits[0] = q;
    p.ph = f.neg ? cd(-1, 0) : eff(0);
    seq.push_back(p);
    return true;
  }
  if (f.type != MOP_U1 || f.nctrl != 0 || f.nb != 1) return false;
  const cd E[4] = {eff(0), eff(1), eff(2), eff(3)};
  cd g, A, B;
  double mt, sn;
  if (!decompose_u2(E, &g, &A, &B, &mt, &sn)) return false;
  FOp pb;
  pb.merge = true;
  pb.bits[0] = q;
  pb.ph = B;
  pb.glob = g;
  seq.push_back(pb);
  FOp r;
  r.type = MOP_LIFT;
  r.nb = 1;
  r.bits[0] = q;
  r.tgt[0] = q;
  r.ntgt = 1;
  r.cls = CLS_DENSE;
  r.off[0] = xtab_push(xt, make_double2(mt, sn));
  finalize_masks(r);
  seq.push_back(r);
  FOp pa;
  pa.merge = true;
  pa.bits[0] = q;
  pa.ph = A;
  seq.push_back(pa);
  return true;
}

// Bind-time fusion (forward schedules): every maximal run of ops that act only on qubit q (pure:
// bit q; density matrices: bits q and q + n) and that no other op on q interrupts becomes one
// 2x2 (pure) or 4x4 (density) op placed at the run's last member (the ops it passes act on other
// qubits and commute with the run). Runs of fixed ops are multiplied here; runs with a
// parametric member get a FuseRec that k_fuse evaluates per sample after binding. Density-matrix
// runs are fused only when they hold a channel or three or more ops (two gate halves cost the
// same as one 4x4, and fixed halves are cheaper split).
static void fuse_runs(mb_circuit c, std::vector<FOp>& seq, int n, bool dm, Schedule* S) {
  const int nq = n;
  std::vector<std::vector<int>> open(nq);
  std::vector<char> drop(seq.size(), 0);
  std::vector<std::pair<int, FOp>> repl;
  auto anchor_mask = [&](int q) { return (uint64_t(1) << q) | (dm ? uint64_t(1) << (q + n) : 0); };
  auto fusable = [&](const FOp& f, int* q) {
    int b = -1;
    switch (f.type) {
      case MOP_U1: case MOP_RROT: case MOP_IROT: case MOP_CTRLX: b = f.nctrl == 0 ? f.tgt[0] : -1; break;
      case MOP_DIAG: b = f.nb == 1 ? f.bits[0] : -1; break;
      case MOP_CPHASE: b = f.nctrl == 1 ? f.ctrl[0] : -1; break;
      case MOP_U2:
        if (dm && f.nb == 2 && f.bits[1] == f.bits[0] + n && f.bits[0] < n) {
          *q = f.bits[0];
          return true;
        }
        return false;
      default: return false;
    }
    if (b < 0) return false;
    *q = dm ? (b < n ? b : b - n) : b;
    return *q >= 0 && *q < nq;
  };
  auto close = [&](int q) {
    std::vector<int>& g = open[q];
    bool channel = false, param = false;
    for (int i : g) {
      channel |= seq[i].type == MOP_U2;
      param |= seq[i].param != 0;
    }
    const bool worth = dm ? (channel || g.size() >= 3) : g.size() >= 2;
    if (!worth) {
      g.clear();
      return;
    }
    const int d = dm ? 4 : 2;
    FuseRec rec{0, d, int(S->fcomps.size()), 0};
    std::vector<FuseComp> comps;
    for (int i : g) {
      const FOp& m = seq[i];
      FuseComp fc{};
      fc.conj = int8_t(m.conj);
      fc.param = int8_t(m.param);
      fc.bit = int8_t(dm && m.type != MOP_U2 && m.bits[0] >= n ? 1 : 0);
      if (m.type == MOP_U2) {
        fc.kind = FC_DENSE4;
        for (int e = 0; e < 16; ++e) fc.off[e] = m.off[e];
      } else if (m.type == MOP_DIAG) {
        fc.kind = FC_DIAG2;
        fc.active = uint8_t(m.active);
        fc.off[0] = m.off[0];
        fc.off[1] = m.off[1];
      } else if (m.type == MOP_CPHASE) {
        fc.kind = FC_PHASE2;
        fc.neg = int8_t(m.neg);
        fc.off[0] = m.off[0];
      } else {
        fc.kind = FC_DENSE2;
        for (int e = 0; e < 4; ++e) fc.off[e] = m.off[e];
      }
      comps.push_back(fc);
    }
    rec.nc = int(comps.size());
    FOp f;
    f.cls = CLS_DENSE;
    if (dm) {
      f.type = MOP_U2;
      f.nb = 2;
      f.bits[0] = f.tgt[0] = q;
      f.bits[1] = f.tgt[1] = q + n;
      f.ntgt = 2;
    } else {
      f.type = MOP_U1;
      f.nb = 1;
      f.bits[0] = f.tgt[0] = q;
      f.ntgt = 1;
    }
    if (param) {
      rec.out = S->xrow;
      S->xrow += d * d;
      S->fcomps.insert(S->fcomps.end(), comps.begin(), comps.end());
      S->frecs.push_back(rec);
      for (int e = 0; e < d * d; ++e) f.off[e] = (rec.out + e) | kXtabFlag;
      f.param = 1;
    } else {
      rec.c0 = 0;
      double2 M[16];
      fuse_product(rec, comps.data(), c->fixed_table.data(), c->fixed_table.data(), M);
      for (int e = 0; e < d * d; ++e) f.off[e] = xtab_push(&S->xtab, M[e]);
    }
    finalize_masks(f);
    for (size_t k = 0; k + 1 < g.size(); ++k) drop[g[k]] = 1;
    repl.push_back({g.back(), f});
    g.clear();
  };
  for (size_t i = 0; i < seq.size(); ++i) {
    int q;
    if (fusable(seq[i], &q)) {
      open[q].push_back(int(i));
      continue;
    }
    for (int a = 0; a < nq; ++a)
      if (!open[a].empty() && (seq[i].all & anchor_mask(a))) close(a);
  }
  for (int a = 0; a < nq; ++a)
    if (!open[a].empty()) close(a);
  for (auto& r : repl) seq[r.first] = r.second;
  std::vector<FOp> out;
  out.reserve(seq.size());
  for (size_t i = 0; i < seq.size(); ++i)
    if (!drop[i]) out.push_back(seq[i]);
  seq.swap(out);
}

// S: the schedule being built; when given (forward schedules), single-qubit runs are fused at
// bind time and fixed single-qubit ops are split into phases and shear rotations, with the
// phases merged.
// Fixed single-qubit channel supermatrices on a density matrix's (row q, column q + n) pair
// whose entries are real with the population/coherence pattern of depolarizing, amplitude
// damping and dephasing channels (and of their products, inverses and adjoints) run as
// MOP_CHAN: populations mix through a real 2x2, coherences scale by real factors, 12 real
// multiply-adds per 4 amplitudes instead of 64 for a dense complex 4x4.
static void chan_forms(mb_circuit c, std::vector<FOp>& seq, int n, const std::vector<double2>* xt) {
  static const int keep[6] = {0, 12, 5, 10, 3, 15};  // (0,0) (0,3) (1,1) (2,2) (3,0) (3,3), column-major
  for (FOp& f : seq) {
    if (f.type != MOP_U2 || f.param || f.nb != 2 || f.tgt[0] >= n || f.tgt[1] != f.tgt[0] + n) continue;
    bool ok = true;
    for (int e = 0; e < 16 && ok; ++e) {
      const int o = f.off[e];
      double2 x;
      if (o & kXtabFlag) {
        const size_t i = size_t(o & ~kXtabFlag);
        if (!xt || i >= xt->size()) {
          ok = false;
          break;
        }
        x = (*xt)[i];
      } else {
        if (o < 0 || size_t(o) >= c->fixed_table.size()) {
          ok = false;
          break;
        }
        x = c->fixed_table[size_t(o)];
      }
      const bool in = e == 0 || e == 12 || e == 5 || e == 10 || e == 3 || e == 15;
      if (x.y != 0.0 || (!in && x.x != 0.0)) ok = false;
    }
    if (!ok) continue;
    int no[6];
    for (int k = 0; k < 6; ++k) no[k] = f.off[keep[k]];
    std::memset(f.off, 0, sizeof(f.off));
    for (int k = 0; k < 6; ++k) f.off[k] = no[k];
    f.type = MOP_CHAN;
    f.conj = 0;
  }
}

static void build_fops(mb_circuit c, int n, int dm, bool dagger, std::vector<FOp>& out, int lo = 0, int hi = -1,
                       Schedule* S = nullptr) {
  out.clear();
  std::vector<FOp> seq;
  if (hi < 0) hi = int(c->ops.size());
  seq.reserve(size_t(std::max(0, hi - lo)) * (dm ? 2 : 1));
  if (dagger) S = nullptr;
  for (int oi = lo; oi < hi; ++oi) {
    const COp& op = c->ops[oi];
    if (op.kind == MB_OP_CHANNEL) {
      FOp f;
      f.nb = 2 * op.k;
      for (int j = 0; j < op.k; ++j) {
        f.bits[j] = op.pos[j];
        f.bits[j + op.k] = op.pos[j] + n;
      }
      f.mat_off = op.mat_off;
      f.d = 1 << f.nb;
      f.cls = CLS_DENSE;
      f.mode = dagger ? MAT_ADJOINT : MAT_PLAIN;
      if (op.k == 1) {
        f.type = MOP_U2;
        for (int r = 0; r < 4; ++r)
          for (int cc = 0; cc < 4; ++cc) f.off[r + 4 * cc] = dagger ? op.mat_off + cc + 4 * r : op.mat_off + r + 4 * cc;
        f.conj = dagger ? 1 : 0;
        f.tgt[0] = f.bits[0];
        f.tgt[1] = f.bits[1];
        f.ntgt = 2;
        finalize_masks(f);
      }
      seq.push_back(f);
      continue;
    }
    seq.push_back(gate_fop(c, op, 0, 0, dagger));
    if (dm) seq.push_back(gate_fop(c, op, n, 1, dagger));
  }
  for (FOp& f : seq) mark_unfusable_masks(f);
  if (dagger) std::reverse(seq.begin(), seq.end());
  if (S) {
    if (S->fuse && !getenv("MB_NO_FUSE")) fuse_runs(c, seq, n, dm, S);
    if (!getenv("MB_NO_SPLIT")) {
      std::vector<FOp> split;
      split.reserve(seq.size() * 3);  // a fixed 2x2 splits into up to three ops
      for (FOp& f : seq)
        if (!split_fixed_1q(c, f, dm, &S->xtab, split)) split.push_back(std::move(f));
      merge_phases(split, dm, &S->xtab);
      seq.swap(split);
    }
  }
  if (dm && !getenv("MB_NO_CHAN")) chan_forms(c, seq, n, S ? &S->xtab : nullptr);
  out.swap(seq);
}

// Reverse sweep of a pure-state circuit range: U' of every gate in reverse order, each active
// parameter followed by its gradient accumulator (generator D in ordered form at gen_off).
// Inverse of a 4x4 complex matrix (column-major) by Gauss-Jordan elimination with partial
// pivoting; false when singular.
static bool invert4(const cd* M, cd* inv) {
  cd a[4][8];
  for (int r = 0; r < 4; ++r)
    for (int c2 = 0; c2 < 4; ++c2) {
      a[r][c2] = M[r + 4 * c2];
      a[r][c2 + 4] = r == c2 ? cd(1, 0) : cd(0, 0);
    }
  for (int col = 0; col < 4; ++col) {
    int piv = col;
    for (int r = col + 1; r < 4; ++r)
      if (std::abs(a[r][col]) > std::abs(a[piv][col])) piv = r;
    if (!(std::abs(a[piv][col]) > 1e-300)) return false;
    if (piv != col)
      for (int k = 0; k < 8; ++k) std::swap(a[piv][k], a[col][k]);
    const cd d = a[col][col];
    for (int k = 0; k < 8; ++k) a[col][k] /= d;
    for (int r = 0; r < 4; ++r)
      if (r != col) {
        const cd f = a[r][col];
        for (int k = 0; k < 8; ++k) a[r][k] -= f * a[col][k];
      }
  }
  for (int r = 0; r < 4; ++r)
    for (int c2 = 0; c2 < 4; ++c2) inv[r + 4 * c2] = a[r][c2 + 4];
  return true;
}

// Spectral norm of a 4x4 complex matrix (power iteration on A'A).
static double norm2_4(const cd* A) {
  cd v[4] = {1, 0.5, 0.25, 0.125};
  double s = 0;
  for (int it = 0; it < 100; ++it) {
    cd w[4], u[4];
    for (int r = 0; r < 4; ++r) {
      w[r] = 0;
      for (int k = 0; k < 4; ++k) w[r] += A[r + 4 * k] * v[k];
    }
    for (int r = 0; r < 4; ++r) {
      u[r] = 0;
      for (int k = 0; k < 4; ++k) u[r] += std::conj(A[k + 4 * r]) * w[k];
    }
    double nu = 0;
    for (int r = 0; r < 4; ++r) nu += std::norm(u[r]);
    nu = std::sqrt(nu);
    if (!(nu > 0)) return 0;
    for (int r = 0; r < 4; ++r) v[r] = u[r] / nu;
    s = std::sqrt(nu);
  }
  return s;
}

// Growth of rounding errors in y when the reverse sweep uncomputes through instruction op:
// 1 for gates (unitary), ||S^-1||_2 for a single-qubit channel, infinity when it cannot be
// inverted.
double growth_of(mb_circuit c, const COp& op) {
  if (op.kind != MB_OP_CHANNEL) return 1.0;
  if (op.k != 1) return INFINITY;
  cd S[16], inv[16];
  for (int e = 0; e < 16; ++e) S[e] = cd(c->fixed_table[op.mat_off + e].x, c->fixed_table[op.mat_off + e].y);
  if (!invert4(S, inv)) return INFINITY;
  return norm2_4(inv);
}

// Gradient micro-op of one active parameter on the bits of `shift` (0: pure state or the row
// bits; n: the column bits of a density matrix, where the generator enters conjugated).
static FOp grad_fop(const COp& op, int shift) {
  FOp g;
  g.type = MOP_GRAD;
  g.nb = op.k;
  for (int j = 0; j < op.k; ++j) g.bits[j] = op.pos[j] + shift;
  g.ntgt = op.k;
  for (int j = 0; j < op.k; ++j) g.tgt[j] = g.bits[j];
  const int d = 1 << op.k;
  for (int r = 0; r < d; ++r)
    for (int cc = 0; cc < d; ++cc) g.off[r + d * cc] = op.gen_off + r + d * cc;
  g.param = op.parametric ? 1 : 0;
  g.conj = shift ? 1 : 0;
  g.slot = op.slot;
  if (op.k == 1 && op.parametric) {
    // Rotation families have constant generators (k_bind's family_matrix): no table reads
    // and four multiply-adds per pair instead of a 2x2 apply and a dot product. On column bits
    // conj((i/2)X) = -(i/2)X, conj((i/2)Y) = (i/2)Y, conj((i/2)Z) = -(i/2)Z, conj(diag(0,-i))
    // = -diag(0,-i).
    const int code = op.family == MB_FAM_RX ? 1 : op.family == MB_FAM_RY ? 2 : op.family == MB_FAM_RZ ? 3
                     : op.family == MB_FAM_PHASE ? 4 : 0;
    if (code) {
      g.type = MOP_GRADP;
      g.pauli = code;
      g.neg = ((op.flags & MB_OPF_ADJOINT) != 0) != (shift != 0 && code != 2);
      g.conj = 0;
    }
  }
  finalize_masks(g);
  g.nd = g.all;
  return g;
}

// Reverse sweep of a circuit range: U' of every gate in reverse order (on a density matrix: on
// the row bits and conj(U)' on the column bits), each active parameter followed by its gradient
// accumulator (generator D in ordered form at gen_off; density matrices: D on the row bits and
// conj(D) on the column bits, _density_gate_gradient!, circuit.jl:155-172). A single-qubit
// channel S updates delta with S' and uncomputes y with S^-1 (inverted here; the caller bounds
// the error growth with reverse_growth). Returns false when the range has an instruction the
// passes cannot reverse.
static bool build_adjoint_fops(mb_circuit c, int lo, int hi, std::vector<FOp>& out, int dm = 0, int n = 0,
                               std::vector<double2>* xt = nullptr) {
  out.clear();
  for (int oi = hi - 1; oi >= lo; --oi) {
    const COp& op = c->ops[oi];
    if (op.kind == MB_OP_CHANNEL) {
      if (!dm || op.k != 1 || !xt) return false;
      cd S[16], inv[16];
      for (int e = 0; e < 16; ++e) S[e] = cd(c->fixed_table[op.mat_off + e].x, c->fixed_table[op.mat_off + e].y);
      if (!invert4(S, inv)) return false;
      FOp d;
      d.type = MOP_U2;
      d.nb = 2;
      d.bits[0] = d.tgt[0] = op.pos[0];
      d.bits[1] = d.tgt[1] = op.pos[0] + n;
      d.ntgt = 2;
      d.cls = CLS_DENSE;
      for (int r = 0; r < 4; ++r)
        for (int cc = 0; cc < 4; ++cc) d.off[r + 4 * cc] = op.mat_off + cc + 4 * r;  // S' = conj(S^T)
      d.conj = 1;
      d.only = 2;
      finalize_masks(d);
      FOp y = d;
      y.conj = 0;
      y.only = 1;
      for (int e = 0; e < 16; ++e) y.off[e] = xtab_push(xt, make_double2(inv[e].real(), inv[e].imag()));
      out.push_back(d);
      out.push_back(y);
      continue;
    }
    if (op.kind != MB_OP_GATE) return false;
    FOp u = gate_fop(c, op, 0, 0, true);
    mark_unfusable_masks(u);
    out.push_back(u);
    if (dm) {
      FOp uc = gate_fop(c, op, n, 1, true);
      mark_unfusable_masks(uc);
      out.push_back(uc);
    }
    if (op.gen_off >= 0) {
      if (op.k > 2) return false;
      out.push_back(grad_fop(op, 0));
      if (dm) out.push_back(grad_fop(op, n));
    }
  }
  if (dm && !getenv("MB_NO_CHAN")) chan_forms(c, out, n, xt);
  return true;
}

// ---------------------------------------------------------------------------------------------
// Host: pass scheduler
// ---------------------------------------------------------------------------------------------
struct Cand {
  int kind;
  std::vector<int> bits;  // sorted global bits
};

static uint64_t mask_of(const std::vector<int>& b) {
  uint64_t m = 0;
  for (int x : b) m |= uint64_t(1) << x;
  return m;
}

// The scheduler's view of one remaining op: its masks and weight, packed so that scoring a
// candidate bit set scans a small contiguous array.
struct SlimOp {
  uint64_t nd, all;
  float w;
  int fits_any;
};

static float slim_weight(const FOp& f) { return f.type == MOP_DIAG ? 0.25f : (f.type == MOP_U2 ? 2.0f : 1.0f); }

// Score of take_ops for `tmask` (same rule, no list).
static double score_mask(const std::vector<SlimOp>& ops, uint64_t tmask, uint64_t full) {
  uint64_t b_all = 0, b_nd = 0;
  double sc = 0;
  for (const SlimOp& f : ops) {
    const bool fits = f.fits_any && (f.nd & ~tmask) == 0;
    const bool comm = (f.nd & b_all) == 0 && (f.all & b_nd) == 0;
    if (fits && comm) {
      sc += f.w;
    } else {
      b_all |= f.all;
      b_nd |= f.nd;
      if ((b_nd & full) == full) break;
    }
  }
  return sc;
}

// Packs the first (at most 8192) remaining ops, the ones take_ops looks at.
static void slim_ops(const std::vector<FOp>& fops, const std::vector<int>& rem, std::vector<SlimOp>& out) {
  const size_t lim = std::min<size_t>(rem.size(), 8192);
  out.resize(lim);
  for (size_t i = 0; i < lim; ++i) {
    const FOp& f = fops[rem[i]];
    out[i] = {f.nd, f.all, slim_weight(f), f.type != F_UNFUSABLE};
  }
}

// Greedy take: ops that fit `tmask` and commute with every op skipped before them.
static std::vector<int> take_ops(const std::vector<FOp>& fops, const std::vector<int>& rem, uint64_t tmask,
                                 uint64_t full, double* score) {
  std::vector<int> taken;
  uint64_t b_all = 0, b_nd = 0;
  double sc = 0;
  const size_t limit = std::min<size_t>(rem.size(), 8192);
  for (size_t i = 0; i < limit; ++i) {
    const FOp& f = fops[rem[i]];
    const bool fits = f.type != F_UNFUSABLE && (f.nd & ~tmask) == 0;
    const bool comm = (f.nd & b_all) == 0 && (f.all & b_nd) == 0;
    if (fits && comm) {
      taken.push_back(rem[i]);
      sc += slim_weight(f);
    } else {
      b_all |= f.all;
      b_nd |= f.nd;
      if ((b_nd & full) == full) break;
    }
  }
  if (score) *score = sc;
  return taken;
}

// Dimension chunks of a tile's bit set for the TMA tensor map (dim 0 = bits 0..2).
static bool tile_geom(const std::vector<int>& bits, int N, int nsamples, TmaGeom& g) {
  std::vector<std::pair<int, int>> chunks;  // (start, len)
  chunks.push_back({0, 3});
  size_t i = 3;
  while (i < bits.size()) {
    int s = bits[i], len = 1;
    while (i + len < bits.size() && bits[i + len] == s + len && len < 8) ++len;
    chunks.push_back({s, len});
    i += len;
  }
  const int nd = int(chunks.size()) + (nsamples > 1 ? 1 : 0);
  if (nd > 5) return false;
  g.ndims = nd;
  for (size_t d = 0; d < chunks.size(); ++d) {
    const int next = d + 1 < chunks.size() ? chunks[d + 1].first : N;
    g.start[d] = chunks[d].first;
    g.bits[d] = next - chunks[d].first;
    g.boxb[d] = chunks[d].second;
  }
  if (nsamples > 1) {
    g.start[chunks.size()] = -1;
    g.bits[chunks.size()] = 0;
    g.boxb[chunks.size()] = 0;
  }
  return true;
}

// Register stages of a tile pass: every stage loads 2^R amplitudes per thread over R
// tile-local bits and applies the ops whose targets lie among them.
static void plan_stages(const std::vector<FOp>& fops, const std::vector<int>& ops, Pass& p, int R,
                        std::vector<double2>* xt = nullptr) {
  const int t = p.t;
  std::vector<int> loc(64, -1);
  for (int i = 0; i < t; ++i) loc[p.bits[i]] = i;
  auto lmask = [&](uint64_t gm) {
    uint64_t m = 0;
    while (gm) {
      const int g = __builtin_ctzll(gm);
      gm &= gm - 1;
      if (loc[g] >= 0) m |= uint64_t(1) << loc[g];
    }
    return m;
  };
  // Warp bits: a stage of 2^(t-R) threads has t-R-5 warp-index bits. Local bits >= 6 that the
  // fewest ops need in registers are kept as the warp bits of every stage that leaves them out
  // of its registers, so consecutive such stages exchange amplitudes within each warp only
  // (the specialised kernels then end those stages with __syncwarp instead of a CTA barrier).
  const int nw = std::max(0, t - R - 5);
  std::vector<int> wbits;
  if (nw > 0 && t - 6 >= nw) {
    std::vector<std::pair<int, int>> cnt;
    for (int q = 6; q < t; ++q) {
      int c = 0;
      for (int idx : ops) c += int((lmask(fops[idx].nd) >> q) & 1);
      cnt.push_back({c, -q});
    }
    std::sort(cnt.begin(), cnt.end());
    for (int i = 0; i < nw; ++i) wbits.push_back(-cnt[i].second);
    std::sort(wbits.begin(), wbits.end());
  }
  uint64_t wmask = 0;
  for (int q : wbits) wmask |= uint64_t(1) << q;
  std::vector<int> rem = ops;
  while (!rem.empty()) {
    std::vector<int> regs;
    uint64_t rmask = 0, b_all = 0, b_nd = 0;
    for (int idx : rem) {
      const FOp& f = fops[idx];
      const uint64_t need = lmask(f.nd) & ~rmask;
      const bool comm = (lmask(f.nd) & b_all) == 0 && (lmask(f.all & mask_of(p.bits)) & b_nd) == 0;
      if (comm && int(regs.size()) + __builtin_popcountll(need) <= R) {
        for (int q = 0; q < t; ++q)
          if ((need >> q) & 1) regs.push_back(q);
        rmask |= need;
      } else {
        b_all |= lmask(f.all & mask_of(p.bits));
        b_nd |= lmask(f.nd);
      }
      if (int(regs.size()) == R) break;
    }
    // Fill the register set with bank-neutral high bits first, the warp bits last.
    for (int q = t - 1; q >= 0 && int(regs.size()) < R; --q)
      if (!((rmask >> q) & 1) && q >= 6 && !((wmask >> q) & 1)) {
        regs.push_back(q);
        rmask |= uint64_t(1) << q;
      }
    for (int q = 0; q < t && int(regs.size()) < R; ++q)
      if (!((rmask >> q) & 1) && !((wmask >> q) & 1)) {
        regs.push_back(q);
        rmask |= uint64_t(1) << q;
      }
    for (int q : wbits)
      if (int(regs.size()) < R && !((rmask >> q) & 1)) {
        regs.push_back(q);
        rmask |= uint64_t(1) << q;
      }
    // Take the ops that fit. A single-bit diagonal whose bit is a thread bit here is left for a
    // later stage when a later op of the pass acts non-diagonally on that bit (and so brings it
    // into registers): there it multiplies half the amplitudes instead of all of them.
    std::vector<int> taken, left;
    std::vector<uint64_t> later_nd(rem.size() + 1, 0);
    for (size_t i = rem.size(); i-- > 0;) later_nd[i] = later_nd[i + 1] | lmask(fops[rem[i]].nd);
    b_all = b_nd = 0;
    for (size_t ri = 0; ri < rem.size(); ++ri) {
      const int idx = rem[ri];
      const FOp& f = fops[idx];
      const uint64_t nd = lmask(f.nd), al = lmask(f.all & mask_of(p.bits)) | nd;
      const bool comm = (nd & b_all) == 0 && (al & b_nd) == 0;
      const bool diag1 = (f.type == MOP_DIAG && f.nb == 1) || (f.type == MOP_CPHASE && f.nctrl == 1 && !f.neg);
      const bool defer = diag1 && (al & ~rmask) != 0 && (al & ~rmask & later_nd[ri + 1]) != 0;
      if ((nd & ~rmask) == 0 && comm && !defer) {
        taken.push_back(idx);
      } else {
        left.push_back(idx);
        b_all |= al;
        b_nd |= nd;
      }
    }
    // Lanes: three non-register bits among 0..5 with distinct residues mod 3 keep the
    // swizzled shared-memory accesses free of bank conflicts.
    StageDesc sd{};
    sd.nreg = R;
    for (int k = 0; k < R; ++k) sd.reg[k] = regs[k];
    std::vector<int> tidb;
    bool used_res[3] = {false, false, false};
    for (int q = 0; q < 6 && q < t && int(tidb.size()) < 3; ++q)
      if (!((rmask >> q) & 1) && !used_res[q % 3]) {
        tidb.push_back(q);
        used_res[q % 3] = true;
      }
    // the other thread bits ascending; the warp bits last (the top thread-index bits) when this
    // stage holds none of them in registers
    const bool keep_w = !wbits.empty() && (rmask & wmask) == 0;
    for (int q = 0; q < t; ++q)
      if (!((rmask >> q) & 1) && std::find(tidb.begin(), tidb.end(), q) == tidb.end() &&
          !(keep_w && ((wmask >> q) & 1)))
        tidb.push_back(q);
    if (keep_w)
      for (int q : wbits) tidb.push_back(q);
    sd.ntid = int(tidb.size());
    for (int q = 0; q < sd.ntid; ++q) sd.tid[q] = tidb[q];
    sd.op0 = int(p.mops.size());
    auto emit = [&](const FOp& f) {
        MOp m{};
        m.type = int16_t(f.type);
        m.conj = int16_t(f.conj);
        m.param = int16_t(f.param);
        m.only = int16_t(f.only);
        std::memcpy(m.off, f.off, sizeof(m.off));
        auto regidx = [&](int gbit) {
          for (int k = 0; k < R; ++k)
            if (regs[k] == loc[gbit]) return k;
          return -1;
        };
        auto sel = [&](int gbit) { return int16_t(loc[gbit] >= 0 ? loc[gbit] : 64 + gbit); };
        if (f.type == MOP_GRADP) {
          m.nsel = 1;
          m.active = uint32_t(p.grad_slots.size());
          p.grad_slots.push_back(f.slot);
          m.r0 = int16_t(regidx(f.tgt[0]));
          m.r1 = int16_t(f.pauli);
          m.conj = int16_t(f.neg ? 1 : 0);
        } else if (f.type == MOP_GRAD) {
          m.nsel = int16_t(f.nb);
          m.active = uint32_t(p.grad_slots.size());
          p.grad_slots.push_back(f.slot);
          int ra = regidx(f.tgt[0]), rb = f.nb > 1 ? regidx(f.tgt[1]) : -1;
          if (f.nb > 1 && ra > rb) {
            int o2[16];
            const int sw[4] = {0, 2, 1, 3};
            for (int r = 0; r < 4; ++r)
              for (int cc = 0; cc < 4; ++cc) o2[r + 4 * cc] = f.off[sw[r] + 4 * sw[cc]];
            std::memcpy(m.off, o2, sizeof(o2));
            std::swap(ra, rb);
          }
          m.r0 = int16_t(ra);
          m.r1 = int16_t(rb);
        } else if (f.type == MOP_U2) {
          int ra = regidx(f.tgt[0]), rb = regidx(f.tgt[1]);
          if (ra > rb) {
            // swap the local bits of the 4x4 matrix so that local bit 0 is the lower register
            int o2[16];
            const int sw[4] = {0, 2, 1, 3};
            for (int r = 0; r < 4; ++r)
              for (int cc = 0; cc < 4; ++cc) o2[r + 4 * cc] = f.off[sw[r] + 4 * sw[cc]];
            std::memcpy(m.off, o2, sizeof(o2));
            std::swap(ra, rb);
          }
          m.r0 = int16_t(ra);
          m.r1 = int16_t(rb);
        } else if (f.type == MOP_CHAN) {
          m.r0 = int16_t(regidx(f.tgt[0]));  // row bit
          m.r1 = int16_t(regidx(f.tgt[1]));  // column bit
        } else if (f.type == MOP_DIAG) {
          m.nsel = int16_t(f.nb);
          for (int j = 0; j < f.nb; ++j) m.sel[j] = sel(f.bits[j]);
          m.active = f.active;
        } else if (f.type == MOP_CPHASE) {
          m.nsel = int16_t(f.nctrl);
          for (int j = 0; j < f.nctrl; ++j) m.sel[j] = sel(f.ctrl[j]);
          m.r1 = int16_t(f.neg ? 1 : 0);
        } else {
          m.r0 = int16_t(regidx(f.tgt[0]));
          m.nsel = int16_t(f.nctrl);
          for (int j = 0; j < f.nctrl; ++j) m.sel[j] = sel(f.ctrl[j]);
        }
        p.mops.push_back(m);
      };
    // Phases on register bits of this stage are grouped: each phase may move back to just after
    // the last op of the stage that acts non-diagonally on its bit (everything it passes
    // commutes with it), and phases whose windows overlap run as one diagonal over up to three
    // register bits (7 complex multiplies for three phases instead of 12).
    const int T = int(taken.size());
    std::vector<int> wstart(T, -1);
    auto regof = [&](int gbit) {
      for (int k = 0; k < R; ++k)
        if (regs[k] == loc[gbit]) return k;
      return -1;
    };
    if (xt)
      for (int i = 0; i < T; ++i) {
        const FOp& f = fops[taken[i]];
        if (f.type != MOP_CPHASE || f.nctrl != 1 || f.neg || !(f.off[0] & kXtabFlag) || regof(f.ctrl[0]) < 0) continue;
        const int q = f.ctrl[0];
        int st = 0;
        for (int j = i - 1; j >= 0; --j)
          if ((fops[taken[j]].nd >> q) & 1) {
            st = j + 1;
            break;
          }
        wstart[i] = st;
      }
    std::vector<std::vector<int>> group_at(T);
    std::vector<char> grouped(T, 0);
    for (int i = 0; i < T; ++i) {
      if (wstart[i] < 0 || grouped[i]) continue;
      uint64_t bits = 0;
      for (int k = i; k < T && __builtin_popcountll(bits) < 3; ++k) {
        if (wstart[k] < 0 || grouped[k] || wstart[k] > i) continue;
        const int q = fops[taken[k]].ctrl[0];
        if ((bits >> q) & 1) continue;
        bits |= uint64_t(1) << q;
        grouped[k] = 1;
        group_at[i].push_back(k);
      }
    }
    int nemit = 0;
    for (int i = 0; i < T; ++i) {
      const std::vector<int>& g = group_at[i];
      if (g.size() == 1) {
        emit(fops[taken[g[0]]]);
        p.fop_order.push_back(taken[g[0]]);
        ++nemit;
      } else if (g.size() > 1) {
        FOp d;
        d.type = MOP_DIAG;
        d.cls = CLS_DIAG;
        d.nb = int(g.size());
        std::vector<cd> ph(g.size());
        for (size_t j = 0; j < g.size(); ++j) {
          const FOp& f = fops[taken[g[j]]];
          d.bits[j] = f.ctrl[0];
          const double2 v = (*xt)[f.off[0] & ~kXtabFlag];
          ph[j] = cd(v.x, v.y);
          p.fop_order.push_back(taken[g[j]]);
        }
        d.active = ((1u << (1 << d.nb)) - 1) & ~1u;
        for (int a = 1; a < (1 << d.nb); ++a) {
          cd prod(1, 0);
          for (int j = 0; j < d.nb; ++j)
            if ((a >> j) & 1) prod *= ph[j];
          d.off[a] = xtab_push(xt, make_double2(prod.real(), prod.imag()));
        }
        finalize_masks(d);
        emit(d);
        ++nemit;
      }
      if (wstart[i] >= 0) continue;  // a grouped phase: emitted with its group
      emit(fops[taken[i]]);
      p.fop_order.push_back(taken[i]);
      ++nemit;
    }
    sd.nops = nemit;
    p.stages.push_back(sd);
    rem.swap(left);
  }
}

static void encode_reg_pass(const std::vector<FOp>& fops, const std::vector<int>& ops, Pass& p) {
  const int R = p.t;
  StageDesc sd{};
  sd.nreg = R;
  for (int k = 0; k < R; ++k) sd.reg[k] = p.bits[k];
  sd.op0 = 0;
  for (int idx : ops) {
    const FOp& f = fops[idx];
    p.fop_order.push_back(idx);
    MOp m{};
    m.type = int16_t(f.type);
    m.conj = int16_t(f.conj);
    m.param = int16_t(f.param);
    std::memcpy(m.off, f.off, sizeof(m.off));
    auto regidx = [&](int gbit) {
      for (int k = 0; k < R; ++k)
        if (p.bits[k] == gbit) return k;
      return -1;
    };
    if (f.type == MOP_U2) {
      int ra = regidx(f.tgt[0]), rb = regidx(f.tgt[1]);
      if (ra > rb) {
        int o2[16];
        const int sw[4] = {0, 2, 1, 3};
        for (int r = 0; r < 4; ++r)
          for (int cc = 0; cc < 4; ++cc) o2[r + 4 * cc] = f.off[sw[r] + 4 * sw[cc]];
        std::memcpy(m.off, o2, sizeof(o2));
        std::swap(ra, rb);
      }
      m.r0 = int16_t(ra);
      m.r1 = int16_t(rb);
    } else if (f.type == MOP_CHAN) {
      m.r0 = int16_t(regidx(f.tgt[0]));
      m.r1 = int16_t(regidx(f.tgt[1]));
    } else if (f.type == MOP_DIAG) {
      m.nsel = int16_t(f.nb);
      for (int j = 0; j < f.nb; ++j) m.sel[j] = int16_t(f.bits[j]);
      m.active = f.active;
    } else if (f.type == MOP_CPHASE) {
      m.nsel = int16_t(f.nctrl);
      for (int j = 0; j < f.nctrl; ++j) m.sel[j] = int16_t(f.ctrl[j]);
      m.r1 = int16_t(f.neg ? 1 : 0);
    } else {
      m.r0 = int16_t(regidx(f.tgt[0]));
      m.nsel = int16_t(f.nctrl);
      for (int j = 0; j < f.nctrl; ++j) m.sel[j] = int16_t(f.ctrl[j]);
    }
    p.mops.push_back(m);
  }
  sd.nops = int(ops.size());
  p.stages.push_back(sd);
}

static std::vector<int> window(int lo, int len, int N) {
  std::vector<int> w;
  for (int q = lo; q < lo + len && q < N; ++q) w.push_back(q);
  return w;
}

struct SchedChoice {
  int kind;               // PassKind, or -1: no candidate held the first op
  std::vector<int> bits;
};

// Tile choices of earlier schedules by op structure (bounded; a full map is cleared).
static std::mutex g_sched_memo_mu;
static std::map<std::vector<uint64_t>, std::vector<SchedChoice>> g_sched_memo;

static bool sched_memo_find(const std::vector<uint64_t>& sig, std::vector<SchedChoice>* out) {
  std::lock_guard<std::mutex> lk(g_sched_memo_mu);
  auto it = g_sched_memo.find(sig);
  if (it == g_sched_memo.end()) return false;
  *out = it->second;
  return true;
}

static void sched_memo_store(const std::vector<uint64_t>& sig, const std::vector<SchedChoice>& rec) {
  std::lock_guard<std::mutex> lk(g_sched_memo_mu);
  if (g_sched_memo.size() >= 256) g_sched_memo.clear();
  g_sched_memo[sig] = rec;
}

static void build_schedule(Schedule& S, int nsamples, bool allow_reg = true) {
  const int N = S.N, t = std::min(S.t, N), R = S.R;
  const uint64_t full = N >= 64 ? ~uint64_t(0) : ((uint64_t(1) << N) - 1);
  // MB_SCHED_ONE_WINDOW=1 restricts tile candidates to one window above bits 0..2 (for
  // comparisons); by default a tile may hold two.
  static const bool two_windows = !(getenv("MB_SCHED_ONE_WINDOW") && atoi(getenv("MB_SCHED_ONE_WINDOW")));
  std::vector<int> rem(S.fops.size());
  for (size_t i = 0; i < rem.size(); ++i) rem[i] = int(i);
  S.passes.clear();
  // The greedy choices depend only on the ops' masks, kinds and targets and on the shape, so
  // a circuit of the same structure (a fresh host circuit with new angles) replays the tile
  // choices of an earlier schedule instead of scoring candidates again.
  std::vector<uint64_t> sig = {uint64_t(N), uint64_t(t), uint64_t(R), uint64_t(nsamples > 1), uint64_t(S.dm),
                               uint64_t(S.adjoint), uint64_t(allow_reg), uint64_t(two_windows), S.fops.size()};
  for (const FOp& f : S.fops) {
    sig.push_back(uint64_t(uint32_t(f.type)) | (uint64_t(uint32_t(f.ntgt)) << 32));
    sig.push_back(f.nd);
    sig.push_back(f.all);
    sig.push_back(uint64_t(uint32_t(f.tgt[0])) | (uint64_t(uint32_t(f.tgt[1])) << 32));
  }
  std::vector<SchedChoice> replay_v;
  const bool have = sched_memo_find(sig, &replay_v);
  const std::vector<SchedChoice>* replay = have ? &replay_v : nullptr;
  std::vector<SchedChoice> record;
  size_t ri = 0;
  while (!rem.empty()) {
    const FOp& f0 = S.fops[rem[0]];
    if (f0.type == F_UNFUSABLE) {
      Pass p;
      p.kind = PASS_PLAIN;
      p.plain_fop = rem[0];
      p.fop_order.push_back(rem[0]);
      S.passes.push_back(p);
      rem.erase(rem.begin());
      continue;
    }
    std::vector<int> best_taken;
    TmaGeom bg{};
    int ckind = -1;
    std::vector<int> cbits;
    if (replay && ri < replay->size()) {
      const SchedChoice& ch = (*replay)[ri++];
      ckind = ch.kind;
      cbits = ch.bits;
      if (ckind == PASS_TILE) tile_geom(cbits, N, nsamples, bg);
      if (ckind >= 0) best_taken = take_ops(S.fops, rem, mask_of(cbits), full, nullptr);
    } else {
      replay = nullptr;
      std::vector<Cand> cands;
      std::vector<SlimOp> slim;
      cands.push_back({PASS_TILE, window(0, t, N)});
      if (N > t) {
        // first target bit not coverable by the low tile, in circuit order
        int h0 = -1;
        for (int idx : rem) {
          const FOp& f = S.fops[idx];
          for (int j = 0; j < f.ntgt && h0 < 0; ++j)
            if (f.tgt[j] >= t) h0 = f.tgt[j];
          if (h0 >= 0) break;
        }
        if (h0 >= 0) {
          const int w = t - 3;
          for (int lo : {std::min(h0, N - w), std::max(3, h0 - w + 1)}) {
            lo = std::max(3, std::min(lo, N - w));
            std::vector<int> b = {0, 1, 2};
            for (int q : window(lo, w, N)) b.push_back(q);
            cands.push_back({PASS_TILE, b});
          }
          const int rlo = std::max(5, std::min(h0, N - R));
          if (allow_reg && N - 5 >= R) cands.push_back({PASS_REG, window(rlo, R, N)});
          if (two_windows) {
            // Bits 0..2 and two windows [a, a + w1), [b, b + w2) with w1 + w2 = t - 3: one pass
            // can then continue a chain of gates at two places (the tail of one layer's light
            // cone and the head of the next). Every single window of each width is scored with
            // bits 0..2; the best six positions of width w1 are paired with the best six of
            // width t - 3 - w1 (an exhaustive search over all pairs finds tiles of the same
            // quality on the tested circuits at five times the cost).
            if (slim.empty()) slim_ops(S.fops, rem, slim);
            constexpr int kTop = 6;
            std::vector<std::vector<std::pair<double, int>>> top(w + 1);
            for (int ww = 2; ww <= w - 2; ++ww) {
              std::vector<std::pair<double, int>> sc;
              for (int a = 3; a + ww <= N; ++a) {
                const uint64_t m = uint64_t(7) | (((uint64_t(1) << ww) - 1) << a);
                sc.push_back({-score_mask(slim, m, full), a});
              }
              std::sort(sc.begin(), sc.end());
              if (sc.size() > size_t(kTop)) sc.resize(kTop);
              top[ww] = sc;
            }
            for (int w1 = 2; w1 <= w - 2; ++w1) {
              const int w2 = w - w1;
              if (w1 > w2) break;  // pairs (w1, w2) and (w2, w1) give the same tiles
              for (const auto& pa : top[w1])
                for (const auto& pb : top[w2]) {
                  int a = pa.second, la = w1, b = pb.second, lb = w2;
                  if (a > b) {
                    std::swap(a, b);
                    std::swap(la, lb);
                  }
                  if (b < a + la + 1) continue;  // overlapping or touching: not two windows
                  std::vector<int> bb = {0, 1, 2};
                  for (int q : window(a, la, N)) bb.push_back(q);
                  for (int q : window(b, lb, N)) bb.push_back(q);
                  cands.push_back({PASS_TILE, bb});
                }
            }
          }
          if (S.dm) {
            // Paired windows for density matrices: row bits [a, a+w1) and the matching column
            // bits [b, b+w2) (b = a + n), so a channel's supermatrix on (q, q+n) and both halves
            // of a gate fit one tile even when n exceeds a single window.
            const int nq = N / 2, w1 = (t - 3) / 2, w2 = t - 3 - w1, q0 = h0 % nq;
            if (nq - w1 >= 3) {
              for (int a : {q0, q0 - w1 / 2}) {
                a = std::max(3, std::min(a, nq - w1));
                int b = std::max(nq, std::min((q0 < 3 ? 0 : a) + nq, N - w2));
                std::vector<int> bb = {0, 1, 2};
                for (int q : window(a, w1, N)) bb.push_back(q);
                for (int q : window(b, w2, N)) bb.push_back(q);
                cands.push_back({PASS_TILE, bb});
              }
            }
          }
        }
      }
      double best = -1;
      int bi = -1;
      if (slim.empty()) slim_ops(S.fops, rem, slim);
      for (size_t ci = 0; ci < cands.size(); ++ci) {
        double sc = score_mask(slim, mask_of(cands[ci].bits), full);
        if (cands[ci].kind == PASS_REG) sc *= 0.999;  // prefer the wider tile on ties
        if (sc <= best) continue;
        TmaGeom g{};
        if (cands[ci].kind == PASS_TILE && !tile_geom(cands[ci].bits, N, nsamples, g)) continue;
        best = sc;
        bi = int(ci);
        bg = g;
      }
      if (bi >= 0) {
        ckind = cands[bi].kind;
        cbits = cands[bi].bits;
        best_taken = take_ops(S.fops, rem, mask_of(cbits), full, nullptr);
      }
      record.push_back({ckind, cbits});
    }
    if (ckind < 0 || best_taken.empty()) {
      // No candidate holds the first op (its bits lie farther apart than any window): run it
      // by itself with the plain kernel, which always makes progress. The adjoint has no
      // plain form of its gradient ops, so its schedule is refused instead.
      if (S.adjoint) {
        S.unschedulable = true;
        if (!have) sched_memo_store(sig, record);
        return;
      }
      Pass p;
      p.kind = PASS_PLAIN;
      p.plain_fop = rem[0];
      p.fop_order.push_back(rem[0]);
      S.passes.push_back(p);
      rem.erase(rem.begin());
      continue;
    }
    Pass p;
    p.kind = ckind;
    p.bits = cbits;
    p.t = int(p.bits.size());
    p.geom = bg;
    if (p.kind == PASS_TILE) plan_stages(S.fops, best_taken, p, R, S.adjoint ? nullptr : &S.xtab);
    else encode_reg_pass(S.fops, best_taken, p);
    for (const MOp& m : p.mops) p.has_u2 |= m.type == MOP_U2 || m.type == MOP_CHAN;
    S.passes.push_back(p);
    std::vector<int> left;
    size_t k = 0;
    for (int idx : rem) {
      if (k < best_taken.size() && best_taken[k] == idx) ++k;
      else left.push_back(idx);
    }
    rem.swap(left);
  }
  if (!have) sched_memo_store(sig, record);
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    cudaDriverEntryPointQueryResult q;
    void* p = nullptr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  return fn;
}

static int make_tmap(const Pass& p, double2* base, int N, int nsamples, CUtensorMap* map) {
  EncodeTiledFn enc = encode_fn();
  if (!enc) {
    set_error("cuTensorMapEncodeTiled is unavailable");
    return MB_EDEVICE;
  }
  const TmaGeom& g = p.geom;
  cuuint64_t dims[5], strides[4];
  cuuint32_t box[5], estr[5] = {1, 1, 1, 1, 1};
  for (int d = 0; d < g.ndims; ++d) {
    if (g.start[d] < 0) {
      dims[d] = cuuint64_t(nsamples);
      box[d] = 1;
      if (d > 0) strides[d - 1] = cuuint64_t(16) << N;
      continue;
    }
    dims[d] = d == 0 ? (cuuint64_t(2) << g.bits[0]) : (cuuint64_t(1) << g.bits[d]);
    box[d] = d == 0 ? 16u : (1u << g.boxb[d]);
    if (d > 0) strides[d - 1] = cuuint64_t(16) << g.start[d];
  }
  CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, g.ndims, base, dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("cuTensorMapEncodeTiled failed (%d) for a %d-dim tile", int(r), g.ndims);
    return MB_EDEVICE;
  }
  return MB_OK;
}

static int plain_fop_launch(mb_circuit c, const FOp& f, double2* v, int64_t elems, int nsamples, int64_t mstride,
                            cudaStream_t st) {
  Pos p{};
  p.k = f.nb;
  for (int j = 0; j < f.nb; ++j) p.p[j] = f.bits[j];
  const double2* m = c->d_table + f.mat_off;
  const int64_t ms = f.param ? mstride : 0;
  if (f.nb == 0) return MB_EUNSUPPORTED;
  if (f.cls == CLS_DIAG) return launch_diag(v, elems, nsamples, p, m, ms, f.mode, f.pactive, st);
  if (f.cls == CLS_MONO) return launch_monomial(v, elems, nsamples, p, m, ms, f.mode, f.sigma, f.d, st);
  return launch_dense_block(v, elems, nsamples, p, m, ms, f.mode, true, st);
}

// Tile bits and register bits of the fused schedule. MB_TILE_BITS / MB_REG_BITS override
// the defaults (the autotuner sets them per register size).
struct Tuning {
  int t = 12, R = 4;
  int fuse = 1;   // fusion width: 1 = single-qubit runs fused at bind time, 0 = one micro-op per gate
};

std::mutex g_tune_mu;
std::map<int, std::pair<int, int>> g_tuning;  // register bits -> (tile bits, register bits)
std::map<int, int> g_fusion;                   // register bits -> fusion width

// Specialised kernels are used from MB_JIT_MIN_BITS register bits on (default 18); MB_JIT=0
// disables them. Small states keep the interpreter kernels (no compile latency).
std::mutex g_spec_mu;
std::map<int, int> g_specialised;  // register bits -> 1 always / 0 never use the specialised kernels

static bool want_jit(int N) {
  const char* e = getenv("MB_JIT");
  if (e && atoi(e) == 0) return false;
  {
    std::lock_guard<std::mutex> lk(g_spec_mu);
    auto it = g_specialised.find(N);
    if (it != g_specialised.end()) return it->second != 0;
  }
  int lo = 18;
  if (const char* m = getenv("MB_JIT_MIN_BITS")) lo = atoi(m);
  return N >= lo;
}

// Defaults: sizes run by the specialised kernels use the shape below; the interpreter kernels
// use 2^12 tiles with 16 amplitudes per thread. mb_tuning_set / the autotuner override both per
// register size.
static Tuning tuning_for(int N) {
  Tuning tu;
  if (want_jit(N) && jit_available()) {
    // 2^10-amplitude tiles, 8 amplitudes per thread, 4 CTAs of 128 threads per SM: the fastest
    // point of a sweep over (t, R, CTAs) on the 28-qubit U3 + CZ step (62.5 ms against 63.8 ms
    // at 2^11 tiles with 2 CTAs of 256 threads, 67.7 ms at 2^12 with 1 CTA of 512)
    tu.t = 10;
    tu.R = 3;
  }
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tuning.find(N);
    if (it != g_tuning.end()) {
      tu.t = it->second.first;
      tu.R = it->second.second;
    }
    auto fi = g_fusion.find(N);
    if (fi != g_fusion.end()) tu.fuse = fi->second;
  }
  if (const char* e = getenv("MB_TILE_BITS")) tu.t = std::max(8, std::min(12, atoi(e)));
  if (const char* e = getenv("MB_REG_BITS")) tu.R = std::max(3, std::min(5, atoi(e)));
  tu.t = std::min(tu.t, N);
  return tu;
}

}  // namespace

static void prepare_jit(Schedule* S);

double reverse_growth(mb_circuit c, const COp& op) { return growth_of(c, op); }

bool jit_sizes(int nbits) { return want_jit(nbits) && jit_available(); }

// force: a tile and register width to use instead of the tuning table's; tile_only: no
// register passes (every pass a tile pass, for the persistent uneven-batch kernel).
static int get_schedule_impl(mb_circuit c, int n, int dm, int adjoint, int lo, int hi, int nsamples,
                             const Tuning* force, bool tile_only, Schedule** out) {
  const int N = dm ? 2 * n : n;
  if (hi < 0) hi = int(c->ops.size());
  Tuning tu = tuning_for(N);
  if (force) {
    tu.t = std::min(force->t, N);
    tu.R = force->R;
  }
  if (adjoint) {
    // y and delta tiles, double-buffered: MB_ADJOINT_TILE_BITS (8..11) and the register width of
    // the dual-state passes MB_ADJOINT_REG_BITS (3..4). Default 2^10-amplitude tiles, 8
    // amplitudes per thread, 3 CTAs per SM: the fastest point of a sweep on the 24-qubit,
    // 1152-angle gradient (47.8 ms against 60.2 ms at 2^11 tiles, 16 amplitudes, 1 CTA).
    tu.t = std::min(tu.t, 10);
    tu.R = 3;
    if (const char* e = getenv("MB_ADJOINT_TILE_BITS")) tu.t = std::max(8, std::min(11, atoi(e)));
    if (const char* e = getenv("MB_ADJOINT_REG_BITS")) tu.R = std::max(3, std::min(4, atoi(e)));
    tu.t = std::min(tu.t, N);
  }
  // A forward schedule of a batch serves every batch up to its capacity (the passes are the
  // same for all batches of more than one sample; only the per-sample rows of the derived
  // table grow), so batches of varying size, as in the serving loop, share one schedule.
  // Capacities are powers of two; adjoint schedules keep their exact batch.
  int cap = nsamples;
  if (!adjoint && nsamples > 1)
    for (cap = 2; cap < nsamples; cap *= 2) {
    }
  auto fits = [&](const Schedule* s) {
    if (adjoint || nsamples == 1) return s->nsamples == nsamples;
    return s->nsamples > 1 && s->nsamples >= nsamples;
  };
  for (Schedule* s : c->scheds)
    if (s->N == N && s->dm == dm && !s->dagger && s->t == tu.t && s->R == tu.R && fits(s) &&
        (adjoint || s->fuse == (tu.fuse != 0)) &&
        s->lo == lo && s->hi == hi && s->adjoint == adjoint && s->tile_only == tile_only) {
      *out = s;
      return MB_OK;
    }
  nsamples = cap;
  if (g_ctx.capturing) {
    set_error("run this circuit once on a state of this shape before capturing it (schedules are built lazily)");
    return MB_EUNSUPPORTED;
  }
  std::unique_ptr<Schedule> S(new Schedule());
  S->N = N;
  S->dm = dm;
  S->t = tu.t;
  S->R = tu.R;
  S->nsamples = nsamples;
  S->lo = lo;
  S->hi = hi;
  S->adjoint = adjoint;
  S->fuse = tu.fuse != 0;
  if (adjoint) {
    if (!build_adjoint_fops(c, lo, hi, S->fops, dm, n, &S->xtab)) {
      set_error("the fused adjoint supports circuits with 1- and 2-qubit parameters and single-qubit channels");
      return MB_EUNSUPPORTED;
    }
  } else {
    build_fops(c, n, dm, false, S->fops, lo, hi, S.get());
  }
  S->tile_only = tile_only;
  build_schedule(*S, nsamples, !adjoint && !tile_only);
  if (S->unschedulable) {
    set_error("the fused adjoint cannot place an instruction whose qubits are farther apart than a tile");
    return MB_EUNSUPPORTED;
  }
  // Every register op must name register bits inside the stage width.
  for (const Pass& p : S->passes) {
    const int R = p.kind == PASS_REG ? p.t : S->R;
    for (const MOp& m : p.mops) {
      const bool needs = m.type == MOP_U1 || m.type == MOP_CTRL || m.type == MOP_CTRLX || m.type == MOP_U2 ||
                         m.type == MOP_GRAD || m.type == MOP_RROT || m.type == MOP_IROT || m.type == MOP_LIFT ||
                         m.type == MOP_GRADP || m.type == MOP_CHAN;
      const bool two = m.type == MOP_U2 || (m.type == MOP_GRAD && m.nsel == 2);
      const bool chan_bad = m.type == MOP_CHAN && (m.r1 < 0 || m.r1 >= R || m.r1 == m.r0);
      if (needs && (m.r0 < 0 || m.r0 >= R || (two && (m.r1 <= m.r0 || m.r1 >= R)) || chan_bad)) {
        set_error("internal scheduling error: micro-op %d without a register target", int(m.type));
        return MB_EUNSUPPORTED;
      }
    }
  }
  std::vector<StageDesc> st;
  std::vector<MOp> mo;
  std::vector<int> gs;
  for (Pass& p : S->passes) {
    p.stage_off = int(st.size());
    p.mop_off = int(mo.size());
    p.grad_off = int(gs.size());
    for (StageDesc sd : p.stages) {
      sd.op0 += p.mop_off;
      st.push_back(sd);
    }
    mo.insert(mo.end(), p.mops.begin(), p.mops.end());
    gs.insert(gs.end(), p.grad_slots.begin(), p.grad_slots.end());
    S->max_grad = std::max(S->max_grad, int(p.grad_slots.size()));
  }
  int rc;
  if (!st.empty()) {
    if ((rc = dev_alloc((void**)&S->d_stages, sizeof(StageDesc) * st.size()))) return rc;
    MB_CHECK_CUDA(cudaMemcpyAsync(S->d_stages, st.data(), sizeof(StageDesc) * st.size(), cudaMemcpyHostToDevice,
                                  g_ctx.stream));
  }
  if (!mo.empty()) {
    if ((rc = dev_alloc((void**)&S->d_mops, sizeof(MOp) * mo.size()))) return rc;
    MB_CHECK_CUDA(cudaMemcpyAsync(S->d_mops, mo.data(), sizeof(MOp) * mo.size(), cudaMemcpyHostToDevice, g_ctx.stream));
  }
  if (!gs.empty()) {
    if ((rc = dev_alloc((void**)&S->d_gslots, sizeof(int) * gs.size()))) return rc;
    MB_CHECK_CUDA(cudaMemcpyAsync(S->d_gslots, gs.data(), sizeof(int) * gs.size(), cudaMemcpyHostToDevice, g_ctx.stream));
  }
  if (!S->xtab.empty() || S->xrow > 0) {
    // fixed derived entries, then nsamples rows of per-sample fused products
    const size_t total = S->xtab.size() + size_t(S->xrow) * size_t(nsamples);
    if ((rc = dev_alloc((void**)&S->d_xtab, sizeof(double2) * std::max<size_t>(1, total)))) return rc;
    if (!S->xtab.empty())
      MB_CHECK_CUDA(cudaMemcpyAsync(S->d_xtab, S->xtab.data(), sizeof(double2) * S->xtab.size(), cudaMemcpyHostToDevice,
                                    g_ctx.stream));
  }
  if (!S->frecs.empty()) {
    if ((rc = dev_alloc((void**)&S->d_frecs, sizeof(FuseRec) * S->frecs.size()))) return rc;
    if ((rc = dev_alloc((void**)&S->d_fcomps, sizeof(FuseComp) * S->fcomps.size()))) return rc;
    MB_CHECK_CUDA(cudaMemcpyAsync(S->d_frecs, S->frecs.data(), sizeof(FuseRec) * S->frecs.size(), cudaMemcpyHostToDevice,
                                  g_ctx.stream));
    MB_CHECK_CUDA(cudaMemcpyAsync(S->d_fcomps, S->fcomps.data(), sizeof(FuseComp) * S->fcomps.size(),
                                  cudaMemcpyHostToDevice, g_ctx.stream));
  }
  MB_CHECK_CUDA(cudaStreamSynchronize(g_ctx.stream));
  if (!adjoint && !tile_only && S->R == 3 && !getenv("MB_REG_BITS")) {
    // Register width 3 exists only as specialised kernels: if they cannot all be built (source
    // limits, compile budget), use width 4 for this register size from now on. (A width forced
    // through MB_REG_BITS is kept; run_schedule then reports the missing kernels. Tile-only
    // schedules belong to the persistent uneven launch, which compiles its own kernel.)
    prepare_jit(S.get());
    if (S->jit != 1) {
      if (getenv("MB_JIT_VERBOSE")) fprintf(stderr, "mossb200: %d-bit schedules fall back to register width 4\n", N);
      {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tuning[N] = {S->t, 4};
      }
      dev_free(S->d_stages);
      dev_free(S->d_mops);
      dev_free(S->d_gslots);
      dev_free(S->d_xtab);
      dev_free(S->d_frecs);
      dev_free(S->d_fcomps);
      return get_schedule_impl(c, n, dm, adjoint, lo, hi, nsamples, force, tile_only, out);
    }
  }
  *out = S.get();
  c->scheds.push_back(S.release());
  return MB_OK;
}

int get_schedule_ex(mb_circuit c, int n, int dm, int adjoint, int lo, int hi, int nsamples, Schedule** out) {
  return get_schedule_impl(c, n, dm, adjoint, lo, hi, nsamples, nullptr, false, out);
}

int get_schedule(mb_circuit c, int n, int dm, bool dagger, int nsamples, Schedule** out) {
  (void)dagger;
  return get_schedule_ex(c, n, dm, 0, 0, -1, nsamples, out);
}


// CTAs per SM of a specialised tile pass: as many double-buffered tiles as shared memory holds
// (allowing 4 KB for the pass's matrix copy; a larger copy only lowers the resident count),
// capped at MB_TILE_CTAS (default 4 for tiles of at most 2^10 amplitudes, else 2). The kernel's launch bounds ask the compiler to fit that
// many CTAs in the register file.
static int tile_ctas(int t) {
  const size_t shm = (size_t(32) << t) + 1024 + 4 * 1024;
  int cap = t <= 10 ? 4 : 2;
  if (const char* e = getenv("MB_TILE_CTAS")) cap = std::max(1, std::min(8, atoi(e)));
  return std::max(1, std::min(cap, int((227 * 1024) / (shm + 256))));
}

// CTAs per SM of a dual-state adjoint pass: what shared memory holds of four double-buffered
// tiles plus the gradient slots (allowing 8 KB), capped at MB_ADJOINT_CTAS (default 3); the
// kernel's launch bounds ask the compiler to fit that many CTAs in the register file.
static int adjoint_ctas(int t, int dm = 0) {
  const size_t shm = (size_t(64) << t) + 1024 + 8 * 1024;
  int cap = dm ? 2 : 3;  // density passes hold 4x4 channel operators for both states: 2 CTAs keep them unspilled
  if (const char* e = getenv("MB_ADJOINT_CTAS")) cap = std::max(1, std::min(4, atoi(e)));  // gpart holds 4 per SM
  return std::max(1, std::min(cap, int((227 * 1024) / (shm + 256))));
}

// Generated kernel sources, memoised by everything the generators read: the pass (bits, TMA
// geometry, register stages, micro-ops, gradient slots) and the kernel shape. Circuits that
// differ only in matrix values (a fresh host circuit with new angles) lower to passes with the
// same micro-ops and table offsets, so their schedules reuse the source text instead of
// generating it again (about 3 ms for the 28-qubit U3 + CZ circuit's 700 KB).
static std::string pass_key(const Pass& p, int gen, int R, int N, bool single, int ctas) {
  std::string k;
  auto put = [&](const void* d, size_t n) { k.append(static_cast<const char*>(d), n); };
  auto put_i = [&](int64_t v) { put(&v, sizeof v); };
  for (int64_t v : {int64_t(gen), int64_t(R), int64_t(N), int64_t(single), int64_t(ctas), int64_t(p.kind),
                    int64_t(p.t), int64_t(p.has_u2)})
    put_i(v);
  put_i(int64_t(p.bits.size()));
  for (int b : p.bits) put_i(b);
  put_i(p.geom.ndims);
  for (int d = 0; d < 5; ++d) {
    put_i(p.geom.start[d]);
    put_i(p.geom.bits[d]);
    put_i(p.geom.boxb[d]);
  }
  put_i(int64_t(p.stages.size()));
  for (const StageDesc& sd : p.stages) {
    put_i(sd.op0);
    put_i(sd.nops);
    put_i(sd.nreg);
    for (int r = 0; r < kMaxRegBits; ++r) put_i(sd.reg[r]);
    put_i(sd.ntid);
    for (int r = 0; r < 26; ++r) put_i(sd.tid[r]);
  }
  put_i(int64_t(p.mops.size()));
  for (const MOp& m : p.mops) {
    for (int64_t v : {int64_t(m.type), int64_t(m.r0), int64_t(m.r1), int64_t(m.nsel), int64_t(m.sel[0]),
                      int64_t(m.sel[1]), int64_t(m.sel[2]), int64_t(m.sel[3]), int64_t(m.active), int64_t(m.conj),
                      int64_t(m.param), int64_t(m.only)})
      put_i(v);
    put(m.off, sizeof m.off);
  }
  put_i(int64_t(p.grad_slots.size()));
  for (int g : p.grad_slots) put_i(g);
  return k;
}

static std::string memo_source(const std::string& key, const std::function<std::string()>& gen) {
  static std::mutex mu;
  static std::unordered_map<std::string, std::string> memo;
  static size_t bytes = 0;
  {
    std::lock_guard<std::mutex> lk(mu);
    auto it = memo.find(key);
    if (it != memo.end()) return it->second;
  }
  std::string src = gen();
  std::lock_guard<std::mutex> lk(mu);
  if (bytes > (size_t(256) << 20)) {  // bound the memo at 256 MB of keys and sources
    memo.clear();
    bytes = 0;
  }
  bytes += key.size() + src.size();
  memo.emplace(key, src);
  return src;
}

static void prepare_jit(Schedule* S) {
  if (S->jit != 0) return;
  S->jit = -1;
  if ((!want_jit(S->N) && !S->adjoint) || !jit_available()) return;
  std::vector<std::string> src;
  std::vector<Pass*> who;
  // One sample: every thread reads row 0 of the matrix table, so the parametric elements can be
  // staged in shared memory with the fixed ones.
  const bool single = S->nsamples == 1;
  for (Pass& p : S->passes) {
    if (p.kind == PASS_TILE && !S->adjoint) p.ctas = tile_ctas(p.t);
    if (p.kind == PASS_TILE && S->adjoint) {
      p.ctas = adjoint_ctas(p.t, S->dm);
      src.push_back(memo_source(pass_key(p, 1, S->R, S->N, single, p.ctas),
                                [&] { return jit_adjoint_source(p, S->R, S->N, single, p.ctas); }));
    } else if (p.kind == PASS_TILE) {
      src.push_back(memo_source(pass_key(p, 0, S->R, S->N, single, p.ctas),
                                [&] { return jit_tile_source(p, S->R, S->N, single, p.ctas); }));
    } else if (p.kind == PASS_REG) {
      src.push_back(memo_source(pass_key(p, 2, S->R, S->N, single, 0), [&] { return jit_reg_source(p, S->N, single); }));
    } else {
      continue;
    }
    who.push_back(&p);
  }
  std::vector<CUfunction> fns;
  std::string err;
  // Passes whose kernels do not compile within the budget (MB_JIT_BUDGET_S seconds per
  // schedule, default 30), and passes whose generated source exceeds MB_JIT_MAX_SOURCE_KB
  // (default 128 KB; NVRTC time grows faster than the source: 3 s at 97 KB, 17 s at 238 KB), run on the
  // interpreter kernels, which exist for R = 4 and 5; the adjoint and R = 3 schedules need
  // every specialised kernel (an R = 3 schedule that cannot have them is rebuilt with R = 4;
  // the adjoint's size limit is four times larger).
  double budget = 30.0;
  if (const char* e = getenv("MB_JIT_BUDGET_S")) budget = atof(e);
  size_t max_src = size_t(128) << 10;
  if (const char* e = getenv("MB_JIT_MAX_SOURCE_KB")) max_src = size_t(std::max(1, atoi(e))) << 10;
  const bool partial_ok = !S->adjoint && (S->R == 4 || S->R == 5);
  if (S->adjoint) max_src *= 4;  // no interpreter to fall back on: only refuse the extreme ones
  std::vector<std::string> small;
  std::vector<Pass*> small_who;
  for (size_t i = 0; i < src.size(); ++i) {
    if (src[i].size() <= max_src) {
      small.push_back(std::move(src[i]));
      small_who.push_back(who[i]);
    } else if (!partial_ok) {
      if (getenv("MB_JIT_VERBOSE")) fprintf(stderr, "mossb200: JIT disabled: a pass source has %zu bytes\n", src[i].size());
      return;
    }
  }
  if (jit_prepare(small, fns, &err, partial_ok ? budget : 0.0) != MB_OK) {
    if (getenv("MB_JIT_VERBOSE")) fprintf(stderr, "mossb200: JIT disabled for this schedule: %s\n", err.c_str());
    return;
  }
  for (size_t i = 0; i < small_who.size(); ++i) {
    small_who[i]->jit_fn = fns[i];
    if (fns[i]) jit_retain((void*)fns[i]);
  }
  S->jit = 1;
  if (!g_ctx.capturing) jit_trim();
}

int run_schedule(mb_circuit c, Schedule* S, double2* v, int nsamples, int64_t mstride) {
  cudaStream_t st = g_ctx.stream;
  const int N = S->N;
  const int64_t elems = int64_t(1) << N;
  prepare_jit(S);
  if (S->jit != 1 && S->R != 4 && S->R != 5) {
    set_error("register width %d needs the specialised kernels, which are unavailable", S->R);
    return MB_EUNSUPPORTED;
  }
  // Per-sample fused products (one row when every sample shares the parameters).
  double2* xs = S->d_xtab ? S->d_xtab + S->xtab.size() : nullptr;
  const int64_t xrow = mstride ? S->xrow : 0;
  if (!S->frecs.empty()) {
    const int rows = mstride ? nsamples : 1;
    const int64_t work = int64_t(S->frecs.size()) * rows;
    ProfScope ps("k_fuse", 0.0, st);
    k_fuse<<<unsigned((work + 127) / 128), 128, 0, st>>>(S->d_frecs, int(S->frecs.size()), S->d_fcomps, c->d_table,
                                                          mstride, xs, S->xrow, rows);
    MB_LAUNCHED();
  }
  for (const Pass& p : S->passes) {
    int rc = MB_OK;
    if (p.kind == PASS_PLAIN) {
      rc = plain_fop_launch(c, S->fops[p.plain_fop], v, elems, nsamples, mstride, st);
    } else if (p.kind == PASS_TILE) {
      CUtensorMap map;
      if ((rc = make_tmap(p, v, N, nsamples, &map))) return rc;
      TileArgs a{};
      a.t = p.t;
      a.nstages = int(p.stages.size());
      a.ndims = p.geom.ndims;
      for (int d = 0; d < 5; ++d) {
        a.start[d] = p.geom.start[d];
        a.extb[d] = p.geom.bits[d];
      }
      for (int i = 0; i < p.t; ++i) a.bits[i] = p.bits[i];
      a.tiles_per_sample = int64_t(1) << (N - p.t);
      a.ntiles = a.tiles_per_sample * nsamples;
      a.tstride = mstride;
      a.stages = S->d_stages + p.stage_off;
      a.mops = S->d_mops;
      a.table = c->d_table;
      a.xtab = S->d_xtab;
      a.xtabs = xs;
      a.xrow = xrow;
      a.err = g_ctx.flags + 2;
      const int threads = 1 << (p.t - S->R);
      const size_t shm = (size_t(32) << p.t) + 1024;  // two tile buffers + alignment slack
      const int per_sm = std::max(1, int((227 * 1024) / (shm + 256)));
      int64_t grid = std::min<int64_t>(a.ntiles, int64_t(g_ctx.sm_count) * std::min(per_sm, 4));
      if (S->jit == 1 && p.jit_fn && p.ctas > 0) grid = std::min<int64_t>(a.ntiles, int64_t(g_ctx.sm_count) * p.ctas);
      if (S->jit == 1 && p.jit_fn) {
        ProfScope ps("k_tile_pass_jit", 32.0 * double(elems) * nsamples, st,
                     pass_flops_per_amp(p, false) * double(elems) * nsamples);
        rc = jit_launch_tile((CUfunction)p.jit_fn, &map, c->d_table, S->d_xtab, xs, xrow, mstride, a.tiles_per_sample,
                             a.ntiles, a.err, threads, shm, int(grid), st);
        ++launch_counter();
        if (rc) return rc;
        continue;
      }
      ProfScope ps("k_tile_pass", 32.0 * double(elems) * nsamples, st,
                   pass_flops_per_amp(p, false) * double(elems) * nsamples);
      const bool u2 = p.has_u2;
      auto launch = [&](auto kern) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(shm));
        kern<<<dim3(unsigned(grid)), threads, shm, st>>>(map, a);
      };
      if (S->R == 5) u2 ? launch(k_tile_pass<5, true>) : launch(k_tile_pass<5, false>);
      else u2 ? launch(k_tile_pass<4, true>) : launch(k_tile_pass<4, false>);
      MB_LAUNCHED();
    } else {
      RegArgs a{};
      a.nbits = p.t;
      for (int k = 0; k < p.t; ++k) a.reg[k] = p.bits[k];
      a.N = N;
      a.groups = int64_t(1) << (N - p.t);
      a.nsamples = nsamples;
      a.nops = p.stages[0].nops;
      a.tstride = mstride;
      a.mops = S->d_mops + p.mop_off;
      a.table = c->d_table;
      a.xtab = S->d_xtab;
      a.xtabs = xs;
      a.xrow = xrow;
      const int64_t work = a.groups * nsamples;
      const int block = 128;
      const int grid = grid_for(work, block, int64_t(g_ctx.sm_count) * 16);
      if (S->jit == 1 && p.jit_fn) {
        ProfScope ps("k_reg_pass_jit", 32.0 * double(elems) * nsamples, st,
                     pass_flops_per_amp(p, false) * double(elems) * nsamples);
        rc = jit_launch_reg((CUfunction)p.jit_fn, v, c->d_table, S->d_xtab, xs, xrow, mstride, a.groups, nsamples, grid,
                            st);
        ++launch_counter();
        if (rc) return rc;
        continue;
      }
      ProfScope ps("k_reg_pass", 32.0 * double(elems) * nsamples, st,
                   pass_flops_per_amp(p, false) * double(elems) * nsamples);
      if (p.t == 5) p.has_u2 ? k_reg_pass<5, true><<<grid, block, 0, st>>>(v, a)
                             : k_reg_pass<5, false><<<grid, block, 0, st>>>(v, a);
      else p.has_u2 ? k_reg_pass<4, true><<<grid, block, 0, st>>>(v, a) : k_reg_pass<4, false><<<grid, block, 0, st>>>(v, a);
      MB_LAUNCHED();
    }
    if (rc) return rc;
  }
  return MB_OK;
}

// Reverse sweep over an adjoint schedule: U' on y and delta in every pass, gradient
// contributions added into d_grad (one entry per parameter slot), summed over the schedule's
// samples (stored back to back; they share the parameters).
int run_adjoint_schedule(mb_circuit c, Schedule* S, double2* y, double2* d, double* d_grad) {
  cudaStream_t st = g_ctx.stream;
  const int N = S->N;
  const int64_t elems = int64_t(1) << N;
  prepare_jit(S);
  if (S->jit != 1) {
    set_error("the fused adjoint needs the specialised kernels");
    return MB_EUNSUPPORTED;
  }
  const int threads_chk = 1 << (S->t - S->R);
  if (threads_chk < 32) {
    set_error("state too small for the fused adjoint");
    return MB_EUNSUPPORTED;
  }
  double* gpart = nullptr;
  unsigned* gcount = nullptr;
  const int grid_max = g_ctx.sm_count * 4;
  int rc;
  if ((rc = dev_alloc((void**)&gpart, sizeof(double) * std::max(1, S->max_grad) * grid_max))) return rc;
  if ((rc = dev_alloc((void**)&gcount, sizeof(unsigned)))) {
    dev_free(gpart);
    return rc;
  }
  cudaMemsetAsync(gcount, 0, sizeof(unsigned), st);
  const int B = S->nsamples;
  for (const Pass& p : S->passes) {
    if (p.kind == PASS_PLAIN) {
      const FOp& f = S->fops[p.plain_fop];
      if (f.only != 2 && (rc = plain_fop_launch(c, f, y, elems, B, 0, st))) break;
      if (f.only != 1 && (rc = plain_fop_launch(c, f, d, elems, B, 0, st))) break;
      continue;
    }
    CUtensorMap my, md;
    if ((rc = make_tmap(p, y, N, B, &my)) || (rc = make_tmap(p, d, N, B, &md))) break;
    const int threads = 1 << (p.t - S->R);
    const int nw = std::max(1, threads / 32);
    const size_t shm = (size_t(64) << p.t) + 1024 + sizeof(double) * std::max<size_t>(1, p.grad_slots.size() * nw);
    const int per_sm = std::max(1, int((227 * 1024) / (shm + 256)));
    const int64_t tps = int64_t(1) << (N - p.t), ntiles = tps * B;
    const int grid = int(std::min<int64_t>(ntiles, int64_t(g_ctx.sm_count) * std::min(per_sm, std::max(1, p.ctas))));
    ProfScope ps("k_adjoint_pass_jit", 64.0 * double(elems) * B, st, pass_flops_per_amp(p, true) * double(elems) * B);
    rc = jit_launch_adjoint((CUfunction)p.jit_fn, &my, &md, c->d_table, 0, tps, ntiles, g_ctx.flags + 2, gpart, gcount,
                            d_grad, S->d_gslots + p.grad_off, S->d_xtab, threads, shm, grid, st);
    ++launch_counter();
    if (rc) break;
  }
  dev_free(gpart);
  dev_free(gcount);
  return rc;
}

// Adjoint schedule for instructions [lo, hi) with its specialised kernels compiled; fails
// (MB_EUNSUPPORTED) when the range cannot run fused.
int adjoint_prepare(mb_circuit c, int n, int lo, int hi, Schedule** out, int dm, int nsamples) {
  Schedule* S = nullptr;
  int rc = get_schedule_ex(c, n, dm, 1, lo, hi, nsamples, &S);
  if (rc) return rc;
  prepare_jit(S);
  if (S->jit != 1 || (1 << (S->t - S->R)) < 32) {
    set_error("the fused adjoint is unavailable for this circuit");
    return MB_EUNSUPPORTED;
  }
  *out = S;
  return MB_OK;
}

int apply_fused(mb_circuit c, mb_state s, int64_t mrow_stride) {
  const int dm = s->kind == MB_DENSITY || s->kind == MB_BATCH_DENSITY;
  const int N = dm ? 2 * s->n : s->n;
  if (N < 8) return apply_plain(c, s, mrow_stride);
  for (const COp& op : c->ops)
    if (op.kind == MB_OP_GATE && op.k == 0) return apply_plain(c, s, mrow_stride);
  Schedule* S = nullptr;
  int rc = get_schedule(c, s->n, dm, false, s->batch, &S);
  if (rc) return rc;
  return run_schedule(c, S, s->d, s->batch, mrow_stride);
}

void release_schedules(mb_circuit c) {
  for (Schedule* s : c->scheds) {
    for (const Pass& p : s->passes)
      if (p.jit_fn) jit_release(p.jit_fn);
    dev_free(s->d_stages);
    dev_free(s->d_mops);
    dev_free(s->d_gslots);
    dev_free(s->d_xtab);
    dev_free(s->d_frecs);
    dev_free(s->d_fcomps);
    delete s;
  }
  c->scheds.clear();
}

}  // namespace mb

// ---- persistent uneven batch (host side) -------------------------------------------------------
// Groups of pure states of 8..17 qubits whose schedules (2^min(11, n)-amplitude tiles, 4 register
// bits, no register passes) hold every instruction run in one k_uneven launch; other groups
// (larger or density states, plain passes) run through the ordinary per-group path.
struct mb_uneven_s {
  std::vector<mb_circuit> cs;
  std::vector<mb_state> ss;
  std::vector<int> pgroups;              // persistent groups (input indices), largest first
  std::vector<int> fallback;             // the others
  std::vector<mb::Schedule*> scheds;     // per persistent group
  std::vector<mb::UnevenGroup> hgroups;  // descriptors as last uploaded
  std::vector<mb::UnevenPass> hpasses;
  mb::UnevenGroup* d_groups = nullptr;
  mb::UnevenPass* d_passes = nullptr;
  int4* d_items = nullptr;
  unsigned* d_next = nullptr;           // work counter, then one completion counter per sample
  int nsamples = 0;
  int nitems = 0;
  int chunk_bits = 15;                   // work items hold 2^chunk_bits amplitudes of a sample
  int64_t nbind = 0, nfuse = 0;
  bool u2 = false;
  double bytes = 0, flops = 0;           // algorithmic bytes and flops of one launch
  // Specialised form (mbk_uneven): straight-line code per pass, register width 3; null when
  // the interpreter form k_uneven runs.
  void* jit_fn = nullptr;
  int jthreads = 0, jctas = 0;
  size_t jshm = 0;
  mb::UnevenJitGroup* d_jgroups = nullptr;
  int4* d_pinfo = nullptr;
};

namespace mb {
namespace {
// Largest register size in the persistent launch (MB_UNEVEN_MAX_BITS, 8..26; default 17).
int uneven_max_bits() {
  const char* e = getenv("MB_UNEVEN_MAX_BITS");
  return e ? std::max(8, std::min(26, atoi(e))) : 17;
}

// Descriptors from the circuits' current tables and parameters (their device buffers move
// when a larger batch of parameters is staged).
void uneven_descriptors(mb_uneven u, std::vector<UnevenGroup>& out) {
  out.clear();
  int pass0 = 0, sample0 = 0;
  int64_t b0 = 0, f0 = 0;
  for (size_t i = 0; i < u->pgroups.size(); ++i) {
    mb_circuit c = u->cs[u->pgroups[i]];
    mb_state s = u->ss[u->pgroups[i]];
    Schedule* S = u->scheds[i];
    UnevenGroup g{};
    g.n = s->n;
    g.B = s->batch;
    g.pass0 = pass0;
    g.npasses = int(S->passes.size());
    pass0 += g.npasses;
    g.sample0 = sample0;
    sample0 += g.B;
    // chunks of up to 2^chunk_bits amplitudes (the same for every pass of the group: a pass
    // has at least 2^(n - chunk_bits) tiles)
    g.nchunks = int(std::max<int64_t>(1, (int64_t(1) << s->n) >> u->chunk_bits));
    g.bind0 = b0;
    g.fuse0 = f0;
    g.nbinds = int(c->binds.size());
    g.nslots = c->nslots;
    g.binds = c->d_binds;
    g.theta = c->d_theta;
    g.nrecs = int(S->frecs.size());
    g.recs = S->d_frecs;
    g.comps = S->d_fcomps;
    g.states = s->d;
    g.table = c->d_table;
    g.tstride = c->table_elems;
    g.xtab = S->d_xtab;
    g.xtabs = S->d_xtab ? S->d_xtab + S->xtab.size() : nullptr;
    g.xrow = S->xrow;
    b0 += int64_t(g.nbinds) * g.B;
    f0 += int64_t(g.nrecs) * g.B;
    out.push_back(g);
  }
}

bool same_descriptors(const std::vector<UnevenGroup>& a, const std::vector<UnevenGroup>& b) {
  return a.size() == b.size() && (a.empty() || std::memcmp(a.data(), b.data(), sizeof(UnevenGroup) * a.size()) == 0);
}

std::vector<UnevenJitGroup> jit_groups(const std::vector<UnevenGroup>& gs) {
  std::vector<UnevenJitGroup> out;
  for (const UnevenGroup& g : gs)
    out.push_back(UnevenJitGroup{g.states, g.table, g.xtab, g.xtabs, (long long)g.tstride, (long long)g.xrow});
  return out;
}

void uneven_release(mb_uneven u) {
  dev_free(u->d_groups);
  dev_free(u->d_passes);
  dev_free(u->d_items);
  dev_free(u->d_next);
  dev_free(u->d_jgroups);
  dev_free(u->d_pinfo);
  if (u->jit_fn) jit_release(u->jit_fn);
  u->d_groups = nullptr;
  u->d_passes = nullptr;
  u->d_items = nullptr;
  u->d_next = nullptr;
  u->d_jgroups = nullptr;
  u->d_pinfo = nullptr;
  u->jit_fn = nullptr;
}
}  // namespace
}  // namespace mb

extern "C" int mb_uneven_create(const mb_circuit* circuits, const mb_state* states, int ngroups, mb_uneven* out) {
  using namespace mb;
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (int rc = check_init()) return rc;
  if (int rc = check_not_capturing("mb_uneven_create")) return rc;
  if (!out || ngroups < 0 || (ngroups && (!circuits || !states))) return MB_EINVAL;
  std::unique_ptr<mb_uneven_s> u(new mb_uneven_s());
  for (int g = 0; g < ngroups; ++g) {
    if (!circuits[g] || !states[g]) return MB_EINVAL;
    if (int rc = validate_apply(circuits[g], states[g])) return rc;
    u->cs.push_back(circuits[g]);
    u->ss.push_back(states[g]);
  }
  std::vector<int> order(ngroups);
  for (int g = 0; g < ngroups; ++g) order[g] = g;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return u->ss[a]->n > u->ss[b]->n; });
  // Schedules of every group that fits: 2^min(10, n)-amplitude tiles with 3 register bits for
  // the specialised form, 2^min(11, n) with 4 for the interpreter form.
  const int max_bits = uneven_max_bits();
  auto collect = [&](bool jit) -> int {
    u->pgroups.clear();
    u->fallback.clear();
    u->scheds.clear();
    u->hpasses.clear();
    u->u2 = false;
    u->bytes = u->flops = 0;
    for (int g : order) {
      mb_circuit c = u->cs[g];
      mb_state s = u->ss[g];
      bool ok = (s->kind == MB_PURE || s->kind == MB_BATCH_PURE) && s->n >= 8 && s->n <= max_bits &&
                s->batch > 0;
      for (const COp& op : c->ops)
        if (op.kind == MB_OP_GATE && op.k == 0) ok = false;
      Schedule* S = nullptr;
      if (ok) {
        Tuning f;
        f.t = std::min(jit ? kUnevenJitTile : kUnevenMaxTile, s->n);
        f.R = jit ? 3 : 4;
        if (int rc = get_schedule_impl(c, s->n, 0, 0, 0, -1, s->batch, &f, true, &S)) return rc;
        for (const Pass& p : S->passes) ok = ok && p.kind == PASS_TILE && p.t <= f.t && p.t >= f.R + 1;
        ok = ok && S->R == f.R;
      }
      if (!ok) {
        u->fallback.push_back(g);
        continue;
      }
      u->pgroups.push_back(g);
      u->scheds.push_back(S);
      for (const Pass& p : S->passes) {
        UnevenPass up{};
        up.t = p.t;
        up.nstages = int(p.stages.size());
        for (int q = 0; q < p.t; ++q) up.bits[q] = p.bits[q];
        up.stages = S->d_stages + p.stage_off;
        up.mops = S->d_mops;
        u->hpasses.push_back(up);
        u->u2 = u->u2 || p.has_u2;
        const double amps = double(int64_t(1) << s->n) * s->batch;
        u->bytes += 32.0 * amps;
        u->flops += pass_flops_per_amp(p, false) * amps;
      }
    }
    return MB_OK;
  };
  int rc;
  const char* ej = getenv("MB_UNEVEN_JIT");
  bool jit = jit_available() && !(ej && atoi(ej) == 0);
  // Chunks of the specialised form hold 2^12 amplitudes (four tiles), so even the largest
  // sample's pass spreads over many CTAs; the interpreter form keeps 2^15 (MB_UNEVEN_CHUNK_BITS
  // overrides either, 10..20).
  auto chunk_bits = [&](bool j) {
    const char* e = getenv("MB_UNEVEN_CHUNK_BITS");
    return e ? std::max(10, std::min(20, atoi(e))) : (j ? 12 : 15);
  };
  u->chunk_bits = chunk_bits(jit);
  if ((rc = collect(jit))) return rc;
  if (jit && !u->pgroups.empty()) {
    // one module with a device function per pass of every persistent group
    std::vector<UnevenJitPass> jp;
    for (size_t i = 0; i < u->pgroups.size(); ++i) {
      const int n = u->ss[u->pgroups[i]]->n;
      const Schedule* S = u->scheds[i];
      for (size_t k = 0; k < S->passes.size(); ++k)
        jp.push_back(UnevenJitPass{&S->passes[k], n, k == 0,
                                   int(std::max<int64_t>(1, (int64_t(1) << n) >> u->chunk_bits))});
    }
    size_t shm = 0;
    int threads = 0;
    const size_t need = (size_t(16) << kUnevenJitTile) + 16 * 2048 + 1024;
    u->jctas = std::max(1, std::min(4, int((227 * 1024) / need)));
    std::vector<std::string> src{jit_uneven_source(jp, 3, u->jctas, &threads, &shm)};
    std::vector<CUfunction> fns;
    std::string err;
    if (jit_prepare(src, fns, &err, 0.0) == MB_OK && fns[0]) {
      u->jit_fn = (void*)fns[0];
      jit_retain(u->jit_fn);
      u->jthreads = threads;
      u->jshm = shm;
    } else {
      if (getenv("MB_JIT_VERBOSE")) fprintf(stderr, "mossb200: persistent launch interpreted: %s\n", err.c_str());
      jit = false;
      u->chunk_bits = chunk_bits(false);
      if ((rc = collect(false))) return rc;
    }
  } else {
    jit = false;
  }
  uneven_descriptors(u.get(), u->hgroups);
  // items by pass index first (every chunk of pass p of every sample before any of pass p+1),
  // then largest groups first; the specialised form names the pass by its index over all
  // groups and finds the counters and the group through pinfo
  std::vector<int4> items, pinfo;
  int maxp = 0;
  for (const UnevenGroup& g : u->hgroups) maxp = std::max(maxp, g.npasses);
  for (int pi = 0; pi < maxp; ++pi)
    for (size_t i = 0; i < u->hgroups.size(); ++i) {
      const UnevenGroup& g = u->hgroups[i];
      if (pi >= g.npasses) continue;
      for (int b = 0; b < g.B; ++b)
        for (int ch = 0; ch < g.nchunks; ++ch)
          items.push_back(jit ? make_int4(g.pass0 + pi, b, ch, 0) : make_int4(int(i), b, pi, ch));
    }
  for (size_t i = 0; i < u->hgroups.size(); ++i) {
    const UnevenGroup& g = u->hgroups[i];
    for (int pi = 0; pi < g.npasses; ++pi) pinfo.push_back(make_int4(g.sample0, pi * g.nchunks, int(i), 0));
  }
  u->nitems = int(items.size());
  for (const UnevenGroup& g : u->hgroups) u->nsamples += g.B;
  for (const UnevenGroup& g : u->hgroups) {
    u->nbind += int64_t(g.nbinds) * g.B;
    u->nfuse += int64_t(g.nrecs) * g.B;
  }
  if (!u->pgroups.empty()) {
    if ((rc = dev_alloc((void**)&u->d_groups, sizeof(UnevenGroup) * u->hgroups.size())) ||
        (rc = dev_alloc((void**)&u->d_passes, sizeof(UnevenPass) * std::max<size_t>(1, u->hpasses.size()))) ||
        (rc = dev_alloc((void**)&u->d_items, sizeof(int4) * items.size())) ||
        (rc = dev_alloc((void**)&u->d_next, sizeof(unsigned) * (1 + size_t(u->nsamples)))) ||
        (u->jit_fn && (rc = dev_alloc((void**)&u->d_jgroups, sizeof(UnevenJitGroup) * u->hgroups.size()))) ||
        (u->jit_fn && (rc = dev_alloc((void**)&u->d_pinfo, sizeof(int4) * pinfo.size())))) {
      uneven_release(u.get());
      return rc;
    }
    cudaStream_t st = g_ctx.stream;
    MB_CHECK_CUDA(cudaMemcpyAsync(u->d_groups, u->hgroups.data(), sizeof(UnevenGroup) * u->hgroups.size(),
                                  cudaMemcpyHostToDevice, st));
    if (u->jit_fn) {
      const std::vector<UnevenJitGroup> jg = jit_groups(u->hgroups);
      MB_CHECK_CUDA(cudaMemcpyAsync(u->d_jgroups, jg.data(), sizeof(UnevenJitGroup) * jg.size(), cudaMemcpyHostToDevice,
                                    st));
      MB_CHECK_CUDA(cudaMemcpyAsync(u->d_pinfo, pinfo.data(), sizeof(int4) * pinfo.size(), cudaMemcpyHostToDevice, st));
      MB_CHECK_CUDA(cudaStreamSynchronize(st));  // jg and pinfo leave scope
    }
    if (!u->hpasses.empty())
      MB_CHECK_CUDA(cudaMemcpyAsync(u->d_passes, u->hpasses.data(), sizeof(UnevenPass) * u->hpasses.size(),
                                    cudaMemcpyHostToDevice, st));
    MB_CHECK_CUDA(cudaMemcpyAsync(u->d_items, items.data(), sizeof(int4) * items.size(), cudaMemcpyHostToDevice, st));
    MB_CHECK_CUDA(cudaStreamSynchronize(st));
  }
  *out = u.release();
  return MB_OK;
}

extern "C" int mb_uneven_info(mb_uneven u, int* persistent_groups, int* fallback_groups, int* samples) {
  std::lock_guard<std::recursive_mutex> lk(mb::g_mu);
  if (!u) return MB_EINVAL;
  if (persistent_groups) *persistent_groups = int(u->pgroups.size());
  if (fallback_groups) *fallback_groups = int(u->fallback.size());
  if (samples) *samples = u->nsamples;
  return MB_OK;
}

extern "C" int mb_uneven_apply(mb_uneven u, int flags) {
  using namespace mb;
  std::lock_guard<std::recursive_mutex> lk(g_mu);
  if (int rc = check_init()) return rc;
  if (!u) return MB_EINVAL;
  cudaStream_t st = g_ctx.stream;
  const bool zero = flags & MB_UNEVEN_ZERO;
  // every group's parameters must be staged on the device, one row per sample
  for (size_t g = 0; g < u->cs.size(); ++g)
    if (u->cs[g]->theta_rows != u->ss[g]->batch && u->ss[g]->batch > 0) {
      set_error("mb_uneven_apply: group %zu has %d staged parameter rows for %d samples", g, u->cs[g]->theta_rows,
                u->ss[g]->batch);
      return MB_EINVAL;
    }
  if (!u->pgroups.empty()) {
    std::vector<UnevenGroup> cur;
    uneven_descriptors(u, cur);
    if (!same_descriptors(cur, u->hgroups)) {
      if (int rc = check_not_capturing("mb_uneven_apply after the circuits' parameter buffers moved")) return rc;
      MB_CHECK_CUDA(cudaMemcpyAsync(u->d_groups, cur.data(), sizeof(UnevenGroup) * cur.size(), cudaMemcpyHostToDevice,
                                    st));
      const std::vector<UnevenJitGroup> jg = jit_groups(cur);
      if (u->jit_fn)
        MB_CHECK_CUDA(cudaMemcpyAsync(u->d_jgroups, jg.data(), sizeof(UnevenJitGroup) * jg.size(),
                                      cudaMemcpyHostToDevice, st));
      MB_CHECK_CUDA(cudaStreamSynchronize(st));
      u->hgroups = cur;
    }
    const int ng = int(u->hgroups.size());
    if (u->nbind) {
      ProfScope ps("k_uneven_bind", 0.0, st);
      k_uneven_bind<<<unsigned((u->nbind + 127) / 128), 128, 0, st>>>(u->d_groups, ng, u->nbind);
      MB_LAUNCHED();
    }
    if (u->nfuse) {
      ProfScope ps("k_uneven_fuse", 0.0, st);
      k_uneven_fuse<<<unsigned((u->nfuse + 127) / 128), 128, 0, st>>>(u->d_groups, ng, u->nfuse);
      MB_LAUNCHED();
    }
    MB_CHECK_CUDA(cudaMemsetAsync(u->d_next, 0, sizeof(unsigned) * (1 + size_t(u->nsamples)), st));
    if (u->jit_fn) {
      const int grid = std::min(u->nitems, g_ctx.sm_count * u->jctas);
      ProfScope ps("mbk_uneven", u->bytes, st, u->flops);
      if (int rc = jit_launch_uneven((CUfunction)u->jit_fn, u->d_jgroups, u->d_pinfo, u->d_items, u->nitems, u->d_next,
                                     u->d_next + 1, zero ? 1 : 0, g_ctx.flags + 2, u->jthreads, u->jshm, grid, st))
        return rc;
      MB_LAUNCHED();
    } else {
      const size_t shm = (size_t(16) << kUnevenMaxTile) + (size_t(8) << kUnevenMaxTile) + 1024;
      const int grid = std::min(u->nitems, g_ctx.sm_count * 2);
      ProfScope ps("k_uneven", u->bytes, st, u->flops);
      auto launch = [&](auto kern) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(shm));
        kern<<<grid, kUnevenThreads, shm, st>>>(u->d_groups, u->d_passes, u->d_items, u->nitems, u->d_next,
                                                u->d_next + 1, zero ? 1 : 0, g_ctx.flags + 2);
      };
      u->u2 ? launch(k_uneven<true>) : launch(k_uneven<false>);
      MB_LAUNCHED();
    }
  }
  for (int g : u->fallback) {
    mb_circuit c = u->cs[g];
    mb_state s = u->ss[g];
    if (s->batch == 0) continue;
    if (zero)
      if (int rc = launch_set_basis(s->d, s->elems, s->batch, 0, st)) return rc;
    if (int rc = bind_launch(c, s->batch)) return rc;
    const int64_t stride = s->kind >= MB_BATCH_PURE ? c->table_elems : 0;
    if (int rc = apply_fused(c, s, stride)) return rc;
  }
  return MB_OK;
}

extern "C" int mb_uneven_free(mb_uneven u) {
  std::lock_guard<std::recursive_mutex> lk(mb::g_mu);
  if (!u) return MB_OK;
  if (mb::g_ctx.init) mb::uneven_release(u);
  delete u;
  return MB_OK;
}

extern "C" int mb_circuit_passes(mb_circuit c, int* npasses) {
  std::lock_guard<std::recursive_mutex> lk(mb::g_mu);
  if (int rc = mb::check_init()) return rc;
  if (!c || !npasses) return MB_EINVAL;
  mb::Schedule* S = nullptr;
  if (c->n < 8) {
    *npasses = int(c->ops.size());
    return MB_OK;
  }
  int rc = mb::get_schedule(c, c->n, 0, false, 1, &S);
  if (rc) return rc;
  *npasses = int(S->passes.size());
  return MB_OK;
}

extern "C" int mb_tuning_set(int nbits, int tile_bits, int reg_bits) {
  if (nbits < 1 || nbits > 40 || tile_bits < 8 || tile_bits > 12 || reg_bits < 3 || reg_bits > 5) {
    mb::set_error("tuning out of range (tile bits 8..12, register bits 3..5)");
    return MB_EINVAL;
  }
  std::lock_guard<std::mutex> lk(mb::g_tune_mu);
  mb::g_tuning[nbits] = {tile_bits, reg_bits};
  return MB_OK;
}

extern "C" int mb_tuning_set_fusion(int nbits, int fusion) {
  if (nbits < 1 || nbits > 40 || fusion < 0 || fusion > 1) {
    mb::set_error("fusion width out of range (0 or 1)");
    return MB_EINVAL;
  }
  std::lock_guard<std::mutex> lk(mb::g_tune_mu);
  mb::g_fusion[nbits] = fusion;
  return MB_OK;
}

extern "C" int mb_tuning_set_specialised(int nbits, int mode) {
  if (nbits < 1 || nbits > 40 || mode < -1 || mode > 1) return MB_EINVAL;
  std::lock_guard<std::mutex> lk(mb::g_spec_mu);
  if (mode < 0) mb::g_specialised.erase(nbits);
  else mb::g_specialised[nbits] = mode;
  return MB_OK;
}

extern "C" int mb_tuning_get_fusion(int nbits, int* fusion) {
  if (!fusion) return MB_EINVAL;
  *fusion = mb::tuning_for(nbits).fuse;
  return MB_OK;
}

extern "C" int mb_tuning_get(int nbits, int* tile_bits, int* reg_bits) {
  if (!tile_bits || !reg_bits) return MB_EINVAL;
  mb::Tuning tu = mb::tuning_for(nbits);
  *tile_bits = tu.t;
  *reg_bits = tu.R;
  return MB_OK;
}

// Host-only view of the fused schedule (no device, no mb_init): builds the circuit's
// instructions and the pass schedule for the given shape and reports its passes. `complete` is
// 1 when every fused op landed in exactly one pass.
extern "C" int mb_schedule_info(const mb_op* ops, size_t nops, int n, int dm, int tile_bits, int reg_bits,
                                int nsamples, int* npasses, int* ntile, int* nreg, int* nplain, int* complete) {
  if ((!ops && nops) || !npasses || !ntile || !nreg || !nplain || !complete) return MB_EINVAL;
  const int N = dm ? 2 * n : n;
  if (n < 1 || N > 40 || tile_bits < 8 || tile_bits > 12 || reg_bits < 3 || reg_bits > 5 || nsamples < 1) {
    mb::set_error("schedule info: n, tile bits (8..12) or register bits (3..5) out of range");
    return MB_EINVAL;
  }
  mb_circuit_s c;
  if (int rc = mb::circuit_compile_host(ops, nops, n, &c)) return rc;
  mb::Schedule S;
  S.N = N;
  S.dm = dm ? 1 : 0;
  S.t = std::min(tile_bits, N);
  S.R = reg_bits;
  S.nsamples = nsamples;
  mb::build_fops(&c, n, S.dm, false, S.fops, 0, -1, &S);
  mb::build_schedule(S, nsamples);
  if (const char* dir = getenv("MB_JIT_DUMP")) {
    // Development aid: the specialised kernel source of every pass (compiled offline to read
    // register and spill counts); with MB_JIT_DUMP_ADJOINT the dual-state passes of the
    // circuit's reverse sweep (pure states) as well.
    if (getenv("MB_JIT_DUMP_ADJOINT")) {
      mb::Schedule A;
      A.N = N;
      A.dm = dm ? 1 : 0;
      A.nsamples = nsamples;
      A.t = std::min(std::min(tile_bits, 10), N);
      A.R = 3;
      if (const char* e = getenv("MB_ADJOINT_REG_BITS")) A.R = std::max(3, std::min(4, atoi(e)));
      A.adjoint = 1;
      if (mb::build_adjoint_fops(&c, 0, int(c.ops.size()), A.fops, A.dm, n, &A.xtab)) {
        mb::build_schedule(A, nsamples, false);
        int j = 0;
        for (mb::Pass& ps : A.passes) {
          if (ps.kind != mb::PASS_TILE) continue;
          const std::string src = mb::jit_adjoint_source(ps, A.R, N, nsamples == 1, mb::adjoint_ctas(ps.t, A.dm));
          char path[512];
          snprintf(path, sizeof(path), "%s/adj_%03d.cu", dir, j++);
          if (FILE* f = fopen(path, "w")) {
            fwrite(src.data(), 1, src.size(), f);
            fclose(f);
          }
        }
      }
    }
    int i = 0;
    for (mb::Pass& ps : S.passes) {
      std::string src;
      if (ps.kind == mb::PASS_TILE) src = mb::jit_tile_source(ps, S.R, N, nsamples == 1, mb::tile_ctas(ps.t));
      else if (ps.kind == mb::PASS_REG) src = mb::jit_reg_source(ps, N, nsamples == 1);
      else continue;
      char path[512];
      snprintf(path, sizeof(path), "%s/pass_%03d.cu", dir, i++);
      if (FILE* f = fopen(path, "w")) {
        fwrite(src.data(), 1, src.size(), f);
        fclose(f);
      }
    }
  }
  int t = 0, r = 0, p = 0;
  size_t covered = 0;
  for (const mb::Pass& ps : S.passes) {
    if (ps.kind == mb::PASS_TILE) ++t;
    else if (ps.kind == mb::PASS_REG) ++r;
    else ++p;
    covered += ps.fop_order.size();
  }
  *npasses = int(S.passes.size());
  *ntile = t;
  *nreg = r;
  *nplain = p;
  *complete = covered == S.fops.size() ? 1 : 0;
  return MB_OK;
}

// ---------------------------------------------------------------------------------------------
// Host-only consistency check of the lowering (diagnostic; no device, no mb_init)
// ---------------------------------------------------------------------------------------------
namespace mb {
namespace {

typedef std::complex<double> hcd;

// The circuit's bound table (one sample), the schedule's fixed derived entries and this
// sample's row of per-sample fused products.
struct HostLowering {
  const double2* tab;
  const std::vector<double2>* xt;
  const std::vector<double2>* xr;
  hcd el(int off, int conj, int param = 0) const {
    const double2 v = (off & kXtabFlag) ? (param ? (*xr)[off & ~kXtabFlag] : (*xt)[off & ~kXtabFlag]) : tab[off];
    return hcd(v.x, conj ? -v.y : v.y);
  }
};

// Applies one fused op to a host vector of 2^N amplitudes.
void host_apply_fop(const HostLowering& L, const FOp& f, std::vector<hcd>& v) {
  const int64_t len = int64_t(v.size());
  auto bit = [](int64_t i, int b) { return int((i >> b) & 1); };
  if (f.type == F_UNFUSABLE) {
    // dense in the fused op's mode on its bits (ordered matrix at mat_off)
    const int k = f.nb, d = 1 << k;
    std::vector<hcd> M(size_t(d) * d);
    for (int r = 0; r < d; ++r)
      for (int q = 0; q < d; ++q) {
        const double2 x = L.tab[f.mat_off + r + q * d];
        hcd e(x.x, x.y);
        if (f.mode == MAT_CONJ) e = std::conj(e);
        M[r + q * d] = e;
      }
    if (f.mode == MAT_ADJOINT || f.mode == MAT_TRANSPOSE) {
      std::vector<hcd> T(M.size());
      for (int r = 0; r < d; ++r)
        for (int q = 0; q < d; ++q) T[r + q * d] = f.mode == MAT_ADJOINT ? std::conj(M[q + r * d]) : M[q + r * d];
      M.swap(T);
    }
    uint64_t mask = 0;
    for (int j = 0; j < k; ++j) mask |= uint64_t(1) << f.bits[j];
    std::vector<hcd> x(d), y(d);
    for (int64_t base = 0; base < len; ++base) {
      if (base & int64_t(mask)) continue;
      for (int a = 0; a < d; ++a) {
        int64_t idx = base;
        for (int j = 0; j < k; ++j)
          if ((a >> j) & 1) idx |= int64_t(1) << f.bits[j];
        x[a] = v[idx];
      }
      for (int r = 0; r < d; ++r) {
        hcd acc = 0;
        for (int q = 0; q < d; ++q) acc += M[r + q * d] * x[q];
        y[r] = acc;
      }
      for (int a = 0; a < d; ++a) {
        int64_t idx = base;
        for (int j = 0; j < k; ++j)
          if ((a >> j) & 1) idx |= int64_t(1) << f.bits[j];
        v[idx] = y[a];
      }
    }
    return;
  }
  auto ctl_ok = [&](int64_t i) {
    for (int j = 0; j < f.nctrl; ++j)
      if (!bit(i, f.ctrl[j])) return false;
    return true;
  };
  switch (f.type) {
    case MOP_U1: case MOP_CTRL: case MOP_CTRLX: case MOP_RROT: case MOP_IROT: case MOP_LIFT: {
      const int t = f.tgt[0];
      hcd m00, m10, m01, m11;
      double mt = 0, sn = 0;
      if (f.type == MOP_CTRLX) {
        m00 = m11 = 0;
        m10 = m01 = 1;
      } else if (f.type == MOP_LIFT) {
        const hcd ts = L.el(f.off[0], 0);
        mt = ts.real();
        sn = ts.imag();
      } else {
        m00 = L.el(f.off[0], f.conj, f.param);
        m10 = L.el(f.off[1], f.conj, f.param);
        m01 = L.el(f.off[2], f.conj, f.param);
        m11 = L.el(f.off[3], f.conj, f.param);
        if (f.type == MOP_RROT) {
          m00 = m00.real(); m10 = m10.real(); m01 = m01.real(); m11 = m11.real();
        } else if (f.type == MOP_IROT) {
          m00 = m00.real(); m11 = m11.real(); m01 = hcd(0, m01.imag()); m10 = hcd(0, m10.imag());
        }
      }
      for (int64_t i = 0; i < len; ++i) {
        if (bit(i, t) || !ctl_ok(i)) continue;
        const int64_t jj = i | (int64_t(1) << t);
        hcd x = v[i], y = v[jj];
        if (f.type == MOP_LIFT) {
          x += mt * y;
          y += sn * x;
          x += mt * y;
          v[i] = x;
          v[jj] = y;
        } else {
          v[i] = m00 * x + m01 * y;
          v[jj] = m10 * x + m11 * y;
        }
      }
      return;
    }
    case MOP_U2: {
      hcd u[16];
      for (int e = 0; e < 16; ++e) u[e] = L.el(f.off[e], f.conj, f.param);
      const int b0 = f.tgt[0], b1 = f.tgt[1];
      for (int64_t i = 0; i < len; ++i) {
        if (bit(i, b0) || bit(i, b1)) continue;
        const int64_t id[4] = {i, i | (int64_t(1) << b0), i | (int64_t(1) << b1), i | (int64_t(1) << b0) | (int64_t(1) << b1)};
        hcd x[4], y[4];
        for (int a = 0; a < 4; ++a) x[a] = v[id[a]];
        for (int r = 0; r < 4; ++r) {
          y[r] = 0;
          for (int q = 0; q < 4; ++q) y[r] += u[r + 4 * q] * x[q];
        }
        for (int a = 0; a < 4; ++a) v[id[a]] = y[a];
      }
      return;
    }
    case MOP_CHAN: {
      double k[6];
      for (int e = 0; e < 6; ++e) k[e] = L.el(f.off[e], 0, f.param).real();
      const int b0 = f.tgt[0], b1 = f.tgt[1];
      for (int64_t i = 0; i < len; ++i) {
        if (bit(i, b0) || bit(i, b1)) continue;
        const int64_t i1 = i | (int64_t(1) << b0), i2 = i | (int64_t(1) << b1), i3 = i1 | i2;
        const hcd x0 = v[i], x3 = v[i3];
        v[i] = k[0] * x0 + k[1] * x3;
        v[i3] = k[4] * x0 + k[5] * x3;
        v[i1] *= k[2];
        v[i2] *= k[3];
      }
      return;
    }
    case MOP_DIAG: {
      for (int64_t i = 0; i < len; ++i) {
        int a = 0;
        for (int j = 0; j < f.nb; ++j) a |= bit(i, f.bits[j]) << j;
        if ((f.active >> a) & 1) v[i] *= L.el(f.off[a], f.conj, f.param);
      }
      return;
    }
    case MOP_CPHASE: {
      const hcd fac = f.neg ? hcd(-1, 0) : L.el(f.off[0], f.conj, f.param);
      for (int64_t i = 0; i < len; ++i)
        if (ctl_ok(i)) v[i] *= fac;
      return;
    }
    default:
      return;
  }
}

// Applies one encoded micro-op of a pass the way the pass kernels do: register index k names
// global bit gbit(reg[k]); a selector below 64 names a pass-local bit (tile passes) or a
// global bit (register sweeps), 64 + b the tile base bit b.
void host_apply_mop(const HostLowering& L, const Pass& p, const StageDesc& sd, const MOp& m, std::vector<hcd>& v) {
  const int64_t len = int64_t(v.size());
  const bool tile = p.kind == PASS_TILE;
  auto gbit_of_reg = [&](int k) { return tile ? p.bits[sd.reg[k]] : sd.reg[k]; };
  auto gbit_of_sel = [&](int sel) { return sel >= 64 ? sel - 64 : (tile ? p.bits[sel] : sel); };
  auto bit = [](int64_t i, int b) { return int((i >> b) & 1); };
  auto el = [&](int e) { return L.el(m.off[e], m.conj, m.param); };
  auto sel_ok = [&](int64_t i) {
    for (int j = 0; j < m.nsel; ++j)
      if (!bit(i, gbit_of_sel(m.sel[j]))) return false;
    return true;
  };
  switch (m.type) {
    case MOP_U1: case MOP_CTRL: case MOP_CTRLX: case MOP_RROT: case MOP_IROT: case MOP_LIFT: {
      const int t = gbit_of_reg(m.r0);
      for (int64_t i = 0; i < len; ++i) {
        if (bit(i, t)) continue;
        if ((m.type == MOP_CTRL || m.type == MOP_CTRLX) && !sel_ok(i)) continue;
        const int64_t jj = i | (int64_t(1) << t);
        hcd x = v[i], y = v[jj];
        if (m.type == MOP_CTRLX) {
          v[i] = y;
          v[jj] = x;
        } else if (m.type == MOP_LIFT) {
          const hcd ts = L.el(m.off[0], 0);
          x += ts.real() * y;
          y += ts.imag() * x;
          x += ts.real() * y;
          v[i] = x;
          v[jj] = y;
        } else {
          hcd m00 = el(0), m10 = el(1), m01 = el(2), m11 = el(3);
          if (m.type == MOP_RROT) {
            m00 = m00.real(); m10 = m10.real(); m01 = m01.real(); m11 = m11.real();
          } else if (m.type == MOP_IROT) {
            m00 = m00.real(); m11 = m11.real(); m01 = hcd(0, m01.imag()); m10 = hcd(0, m10.imag());
          }
          v[i] = m00 * x + m01 * y;
          v[jj] = m10 * x + m11 * y;
        }
      }
      return;
    }
    case MOP_U2: {
      const int b0 = gbit_of_reg(m.r0), b1 = gbit_of_reg(m.r1);
      for (int64_t i = 0; i < len; ++i) {
        if (bit(i, b0) || bit(i, b1)) continue;
        const int64_t id[4] = {i, i | (int64_t(1) << b0), i | (int64_t(1) << b1), i | (int64_t(1) << b0) | (int64_t(1) << b1)};
        hcd x[4], y[4];
        for (int a = 0; a < 4; ++a) x[a] = v[id[a]];
        for (int r = 0; r < 4; ++r) {
          y[r] = 0;
          for (int q = 0; q < 4; ++q) y[r] += el(r + 4 * q) * x[q];
        }
        for (int a = 0; a < 4; ++a) v[id[a]] = y[a];
      }
      return;
    }
    case MOP_CHAN: {
      const int b0 = gbit_of_reg(m.r0), b1 = gbit_of_reg(m.r1);
      double k[6];
      for (int e = 0; e < 6; ++e) k[e] = el(e).real();
      for (int64_t i = 0; i < len; ++i) {
        if (bit(i, b0) || bit(i, b1)) continue;
        const int64_t i1 = i | (int64_t(1) << b0), i2 = i | (int64_t(1) << b1), i3 = i1 | i2;
        const hcd x0 = v[i], x3 = v[i3];
        v[i] = k[0] * x0 + k[1] * x3;
        v[i3] = k[4] * x0 + k[5] * x3;
        v[i1] *= k[2];
        v[i2] *= k[3];
      }
      return;
    }
    case MOP_DIAG: {
      for (int64_t i = 0; i < len; ++i) {
        int a = 0;
        for (int j = 0; j < m.nsel; ++j) a |= bit(i, gbit_of_sel(m.sel[j])) << j;
        if ((m.active >> a) & 1) v[i] *= el(a);
      }
      return;
    }
    case MOP_CPHASE: {
      const hcd fac = m.r1 ? hcd(-1, 0) : el(0);
      for (int64_t i = 0; i < len; ++i)
        if (sel_ok(i)) v[i] *= fac;
      return;
    }
    default:
      return;
  }
}

}  // namespace
}  // namespace mb

// Diagnostic: lowers a fixed (non-parametric) circuit for a state of n qubits (dm: density
// matrix) exactly as a forward schedule does, then applies to one seeded random vector on the
// host (a) every instruction with its compiled matrix and (b) the lowered micro-ops in the order
// the scheduled passes run them. err_ops / err_sched: max |(a) - (b)| for the micro-op sequence
// before scheduling and in the scheduled order. For tests of the host lowering only: it returns
// no amplitudes and needs no device.
extern "C" int mb_lowering_check(const mb_op* ops, size_t nops, int n, int dm, int tile_bits, int reg_bits,
                                 uint64_t seed, double* err_ops, double* err_sched, double* err_mops) {
  if ((!ops && nops) || !err_ops || !err_sched || !err_mops) return MB_EINVAL;
  const int N = dm ? 2 * n : n;
  if (n < 1 || N > 22 || tile_bits < 8 || tile_bits > 12 || reg_bits < 3 || reg_bits > 5) {
    mb::set_error("lowering check: at most 22 amplitude bits, tile bits 8..12, register bits 3..5");
    return MB_EINVAL;
  }
  mb_circuit_s c;
  if (int rc = mb::circuit_compile_host(ops, nops, n, &c)) return rc;
  for (const mb::COp& op : c.ops)
    if (op.k == 0) {
      mb::set_error("lowering check: zero-qubit gates are not lowered");
      return MB_EUNSUPPORTED;
    }
  // Bind the parametric instructions on the host (the code k_bind runs), each at its given value.
  std::vector<double2> tab = c.fixed_table;
  for (const mb::BindRec& rc : c.binds) mb::bind_record(rc, rc.value, tab.data(), tab.data());
  mb::Schedule S;
  S.N = N;
  S.dm = dm ? 1 : 0;
  S.t = std::min(tile_bits, N);
  S.R = reg_bits;
  mb::build_fops(&c, n, S.dm, false, S.fops, 0, -1, &S);
  mb::build_schedule(S, 1);
  // this sample's fused products (what k_fuse writes after binding)
  std::vector<double2> xrow(std::max(1, S.xrow));
  for (const mb::FuseRec& r : S.frecs) {
    double2 M[16];
    mb::fuse_product(r, S.fcomps.data(), tab.data(), tab.data(), M);
    for (int e = 0; e < r.d * r.d; ++e) xrow[r.out + e] = M[e];
  }
  // random start vector
  std::vector<mb::hcd> v0(size_t(1) << N);
  uint64_t st = seed * 0x9E3779B97F4A7C15ull + 1;
  auto rnd = [&] {
    st ^= st << 13; st ^= st >> 7; st ^= st << 17;
    return double(st >> 11) * (1.0 / 9007199254740992.0) - 0.5;
  };
  for (auto& x : v0) x = mb::hcd(rnd(), rnd());
  // (a) the instructions with their compiled (ordered) matrices
  std::vector<mb::hcd> ref = v0;
  for (const mb::COp& op : c.ops) {
    mb::FOp f;
    f.type = -1;  // dense on its bits
    f.mat_off = op.mat_off;
    f.mode = mb::MAT_PLAIN;
    if (op.kind == MB_OP_CHANNEL) {
      f.nb = 2 * op.k;
      for (int j = 0; j < op.k; ++j) { f.bits[j] = op.pos[j]; f.bits[j + op.k] = op.pos[j] + n; }
      mb::host_apply_fop(mb::HostLowering{tab.data(), &S.xtab, &xrow}, f, ref);
      continue;
    }
    f.nb = op.k;
    for (int j = 0; j < op.k; ++j) f.bits[j] = op.pos[j];
    mb::host_apply_fop(mb::HostLowering{tab.data(), &S.xtab, &xrow}, f, ref);
    if (dm) {
      for (int j = 0; j < op.k; ++j) f.bits[j] = op.pos[j] + n;
      f.mode = mb::MAT_CONJ;
      mb::host_apply_fop(mb::HostLowering{tab.data(), &S.xtab, &xrow}, f, ref);
    }
  }
  const mb::HostLowering L{tab.data(), &S.xtab, &xrow};
  std::vector<mb::hcd> a = v0, b = v0, e = v0;
  for (const mb::FOp& f : S.fops) mb::host_apply_fop(L, f, a);
  for (const mb::Pass& p : S.passes)
    for (int idx : p.fop_order) mb::host_apply_fop(L, S.fops[idx], b);
  for (const mb::Pass& p : S.passes) {
    if (p.kind == mb::PASS_PLAIN) {
      mb::host_apply_fop(L, S.fops[p.plain_fop], e);
      continue;
    }
    for (const mb::StageDesc& sd : p.stages)
      for (int q = 0; q < sd.nops; ++q) mb::host_apply_mop(L, p, sd, p.mops[sd.op0 + q], e);
  }
  double ea = 0, eb = 0, ec = 0;
  for (size_t i = 0; i < ref.size(); ++i) {
    ea = std::max(ea, std::abs(a[i] - ref[i]));
    eb = std::max(eb, std::abs(b[i] - ref[i]));
    ec = std::max(ec, std::abs(e[i] - ref[i]));
  }
  *err_ops = ea;
  *err_sched = eb;
  *err_mops = ec;
  return MB_OK;
}
