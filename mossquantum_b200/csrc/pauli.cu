// K4: fused Pauli-string expectation <psi|H|psi> and the adjoint seed H psi.
//
// The reference evaluates one dense local matrix per site key, one state pass per key
// (src/observables/expectation.jl:12-33, backends/cpu/expectations/threaded.jl). Here every
// term is decomposed into Pauli strings P = i^{#Y} X^x Z^z with a complex coefficient, and
// the strings are grouped by their flip mask x. For amplitude index j,
//   <psi|P|psi> = sum_j conj(psi_j) * i^{#Y} (-1)^{|(j^x)&z|} psi_{j^x}.
// A pass reads the state once in tiles of 1024 amplitudes: the five lane bits 0..4 times five
// "register" bits chosen for the pass, staged in shared memory, so every group whose flip mask
// lies in those ten local bits finds its partner amplitude in the tile. The sign of a string
// splits into a tile-base part and a local part: strings whose Z mask avoids the local bits
// give one constant per tile, strings inside the local bits are tabulated once per pass over
// the 1024 local indices, and only strings that straddle both are evaluated per amplitude (a
// couple per pass for nearest-neighbour Hamiltonians). TFIM on n qubits takes ceil((n-5)/5)
// passes instead of 2n-1 key passes.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <complex>
#include <map>
#include <memory>
#include <vector>

#include "internal.h"
#include "jit.h"

namespace mb {

typedef std::complex<double> cdd;
constexpr int kPRMax = 7;                 // register bits per pass: 7 from 24 qubits, else 5
constexpr int kPThreads = 256;
constexpr int kPMaxGroups = 128;          // groups per pass (per-tile constants in shared memory)
constexpr int kPTableMin = 1;             // local strings of a group tabulated from this many on

// Tile of a pass with NR register bits: the lane bits 0..4 and NR register bits, 2^(5+NR)
// amplitudes in shared memory (64 KiB for NR = 7), tile / 256 amplitudes per thread.
template <int NR> struct PShape {
  static constexpr int local = 5 + NR;
  static constexpr int tile = 1 << local;
  static constexpr int per = tile / kPThreads;
};

struct PString {
  uint64_t z;
  double2 c;  // coefficient including i^{#Y}
};

// One flip-mask group of one pass; its strings are stored in the program's own order:
// [k0, k0 + nk) constant per tile, [v0, v0 + nv) straddling, the rest tabulated at `tab`.
struct PGroup {
  uint64_t x;   // flip mask (global bits, all among the pass's local bits)
  int xl;       // flip mask as a local index (bits 0..4 lanes, 5..9 registers)
  int k0, nk;
  int v0, nv;
  int tab;      // offset of the group's table (one entry per local index), or -1
  int herm;     // every string's coefficient without i^{#Y} is real (the group is Hermitian)
  int hb;       // highest set bit of xl (flip groups)
};

struct PPassArgs {
  int n;
  int nr;                 // register bits of the pass's tiles (5 or 7)
  int reg[kPRMax];
  int g0, ngroups;
  const PGroup* groups;
  const PString* strings;
  const double2* tables;
  int64_t tiles_per_sample;
};

struct PauliProgram {
  int n = -1;
  int nr = 5;
  std::vector<PPassArgs> passes;
  PGroup* d_groups = nullptr;
  PString* d_strings = nullptr;
  double2* d_tables = nullptr;
  std::vector<void*> jit;        // per pass: specialised expectation kernel (mbk_pauli) or null
  double2* d_coef = nullptr;     // the observable's string coefficients, for the specialised kernels
};

struct PauliData {
  std::vector<PString> strings;  // grouped by flip mask
  std::vector<std::pair<uint64_t, std::pair<int, int>>> groups;  // x -> [s0, ns)
  std::vector<PauliProgram*> programs;
};

namespace {

// Global bits of local index l: lane bits as they are, register bit k at reg[k].
__host__ __device__ __forceinline__ uint64_t local_bits(int l, const int* reg, int nr) {
  uint64_t o = uint64_t(l & 31);
  for (int k = 0; k < nr; ++k)
    if ((l >> (5 + k)) & 1) o |= uint64_t(1) << reg[k];
  return o;
}

// Tile base: tile index T with zeros inserted at the lane bits and the register bits.
template <int NR>
__device__ __forceinline__ uint64_t tile_base(int64_t T, const int* reg) {
  uint64_t base = uint64_t(T) << 5;
#pragma unroll
  for (int k = 0; k < NR; ++k) {
    const int p = reg[k];
    base = ((base >> p) << (p + 1)) | (base & ((uint64_t(1) << p) - 1));
  }
  return base;
}

// Loads a tile into shared memory (each warp reads 32 consecutive amplitudes) and computes the
// per-tile constants of the pass's groups (descriptors already in shared memory): one warp per
// group, its lanes over the group's constant strings.
template <int NR>
__device__ __forceinline__ void stage_tile(const double2* __restrict__ vs, uint64_t base, const uint64_t* loc,
                                           const PPassArgs& a, const PGroup* gd, double2* tile, double2* kconst) {
#pragma unroll
  for (int k = 0; k < PShape<NR>::per; ++k) tile[threadIdx.x + k * kPThreads] = vs[base | loc[k]];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int gi = warp; gi < a.ngroups; gi += kPThreads / 32) {
    const int k0 = gd[gi].k0, nk = gd[gi].nk;
    double2 kc = cz();
    for (int s = k0 + lane; s < k0 + nk; s += 32) {
      const PString ps = a.strings[s];
      const bool odd = __popcll(base & ps.z) & 1;
      kc.x += odd ? -ps.c.x : ps.c.x;
      kc.y += odd ? -ps.c.y : ps.c.y;
    }
    for (int o = 16; o > 0; o >>= 1) {
      kc.x += __shfl_xor_sync(0xffffffffu, kc.x, o);
      kc.y += __shfl_xor_sync(0xffffffffu, kc.y, o);
    }
    if (lane == 0) kconst[gi] = kc;
  }
}

// Factor of group g at local index l (tile base `base`, local bits `lb`).
__device__ __forceinline__ double2 group_factor(const PGroup& g, const PPassArgs& a, double2 kc, int l,
                                                uint64_t base, uint64_t lb) {
  double2 f = kc;
  if (g.tab >= 0) f = cadd(f, __ldg(a.tables + g.tab + l));
  if (g.nv) {
    const uint64_t k_idx = (base | lb) ^ g.x;
    for (int s = g.v0; s < g.v0 + g.nv; ++s) {
      const PString ps = a.strings[s];
      const bool odd = __popcll(k_idx & ps.z) & 1;
      f.x += odd ? -ps.c.x : ps.c.x;
      f.y += odd ? -ps.c.y : ps.c.y;
    }
  }
  return f;
}

__device__ __forceinline__ void load_groups(const PPassArgs& a, PGroup* gd) {
  for (int gi = threadIdx.x; gi < a.ngroups; gi += kPThreads) gd[gi] = a.groups[a.g0 + gi];
}

// <psi|H|psi> over the groups of one pass. Groups are the outer loop (one descriptor read per
// tile), the thread's amplitudes the inner one. A Hermitian flip group sums over pairs
// (j, j^x) only: conj(psi_j) f(j) psi_{j^x} + conj(psi_{j^x}) f(j^x) psi_j equals
// 2 Re(conj(psi_j) f(j) psi_{j^x}) because f(j^x) = conj(f(j)), so half the amplitudes of the
// tile (local bit hb clear) carry the group. The tile is dynamic shared memory.
template <int NR>
__global__ void __launch_bounds__(kPThreads) k_pauli_pass(const double2* __restrict__ v, const PPassArgs a,
                                                         double2* partials, unsigned* counters, double2* out) {
  constexpr int PER = PShape<NR>::per;
  extern __shared__ double2 pauli_tile[];
  double2* tile = pauli_tile;
  __shared__ double2 kconst[kPMaxGroups];
  __shared__ PGroup gd[kPMaxGroups];
  __shared__ double2 wp[kPThreads / 32];
  __shared__ bool last;
  const int b = blockIdx.y, G = gridDim.x;
  const double2* vs = v + (int64_t(b) << a.n);
  int reg[NR];
#pragma unroll
  for (int k = 0; k < NR; ++k) reg[k] = a.reg[k];
  uint64_t loc[PER];
#pragma unroll
  for (int k = 0; k < PER; ++k) loc[k] = local_bits(threadIdx.x + k * kPThreads, reg, NR);
  load_groups(a, gd);
  __syncthreads();
  double2 acc = cz();
  for (int64_t T = blockIdx.x; T < a.tiles_per_sample; T += G) {
    const uint64_t base = tile_base<NR>(T, reg);
    stage_tile<NR>(vs, base, loc, a, gd, tile, kconst);
    __syncthreads();
    for (int gi = 0; gi < a.ngroups; ++gi) {
      const PGroup g = gd[gi];
      const double2 kc = kconst[gi];
      if (g.xl == 0) {
        // diagonal group: f(j) |psi_j|^2
#pragma unroll
        for (int k = 0; k < PER; ++k) {
          const int l = threadIdx.x + k * kPThreads;
          const double2 amp = tile[l];
          const double2 f = group_factor(g, a, kc, l, base, loc[k]);
          const double p2 = amp.x * amp.x + amp.y * amp.y;
          acc.x = fma(f.x, p2, acc.x);
          acc.y = fma(f.y, p2, acc.y);
        }
      } else if (g.herm) {
        const int hb = g.hb;
#pragma unroll
        for (int k = 0; k < PER / 2; ++k) {
          const int m = threadIdx.x + k * kPThreads;
          const int l = ((m >> hb) << (hb + 1)) | (m & ((1 << hb) - 1));
          const double2 amp = tile[l], p = tile[l ^ g.xl];
          const double2 f = group_factor(g, a, kc, l, base, g.nv ? local_bits(l, reg, NR) : 0);
          // 2 Re(conj(amp) p f)
          const double cr = amp.x * p.x + amp.y * p.y, ci = amp.x * p.y - amp.y * p.x;
          acc.x = fma(2.0 * f.x, cr, fma(-2.0 * f.y, ci, acc.x));
        }
      } else {
#pragma unroll
        for (int k = 0; k < PER; ++k) {
          const int l = threadIdx.x + k * kPThreads;
          const double2 amp = tile[l], p = tile[l ^ g.xl];
          const double2 f = group_factor(g, a, kc, l, base, loc[k]);
          const double2 cp = make_double2(amp.x * p.x + amp.y * p.y, amp.x * p.y - amp.y * p.x);
          acc = cfma(f, cp, acc);
        }
      }
    }
    __syncthreads();
  }
  for (int o = 16; o > 0; o >>= 1) {
    acc.x += __shfl_down_sync(0xffffffffu, acc.x, o);
    acc.y += __shfl_down_sync(0xffffffffu, acc.y, o);
  }
  if ((threadIdx.x & 31) == 0) wp[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double2 s = cz();
    for (int w = 0; w < kPThreads / 32; ++w) s = cadd(s, wp[w]);
    partials[int64_t(b) * G + blockIdx.x] = s;
    __threadfence();
    last = atomicAdd(&counters[b], 1u) == unsigned(G - 1);
  }
  __syncthreads();
  if (last && threadIdx.x == 0) {
    double2 s = cz();
    for (int g = 0; g < G; ++g) s = cadd(s, __ldcg(&partials[int64_t(b) * G + g]));
    out[b] = cadd(__ldcg(&out[b]), s);
    counters[b] = 0;
  }
}

// Seed variant: out (+)= scale * H psi, with (P psi)_j = i^{#Y} (-1)^{|(j^x)&z|} psi_{j^x}.
// Same tiles; the first pass writes, later passes add the groups they hold. The thread's
// amplitudes are taken four at a time (four accumulators), each quarter over all groups.
template <int NR>
__global__ void __launch_bounds__(kPThreads) k_pauli_apply(const double2* __restrict__ v, double2* __restrict__ out,
                                                          const PPassArgs a, double scale, int first) {
  constexpr int PER = PShape<NR>::per;
  constexpr int Q = PER < 4 ? PER : 4;
  extern __shared__ double2 pauli_tile[];
  double2* tile = pauli_tile;
  __shared__ double2 kconst[kPMaxGroups];
  __shared__ PGroup gd[kPMaxGroups];
  const int b = blockIdx.y, G = gridDim.x;
  const double2* vs = v + (int64_t(b) << a.n);
  double2* os = out + (int64_t(b) << a.n);
  int reg[NR];
#pragma unroll
  for (int k = 0; k < NR; ++k) reg[k] = a.reg[k];
  uint64_t loc[PER];
#pragma unroll
  for (int k = 0; k < PER; ++k) loc[k] = local_bits(threadIdx.x + k * kPThreads, reg, NR);
  load_groups(a, gd);
  __syncthreads();
  for (int64_t T = blockIdx.x; T < a.tiles_per_sample; T += G) {
    const uint64_t base = tile_base<NR>(T, reg);
    stage_tile<NR>(vs, base, loc, a, gd, tile, kconst);
    __syncthreads();
#pragma unroll
    for (int k0 = 0; k0 < PER; k0 += Q) {
      double2 r[Q];
#pragma unroll
      for (int k = 0; k < Q; ++k) r[k] = cz();
      for (int gi = 0; gi < a.ngroups; ++gi) {
        const PGroup g = gd[gi];
        const double2 kc = kconst[gi];
#pragma unroll
        for (int k = 0; k < Q; ++k) {
          const int l = threadIdx.x + (k0 + k) * kPThreads;
          r[k] = cfma(group_factor(g, a, kc, l, base, loc[k0 + k]), tile[l ^ g.xl], r[k]);
        }
      }
#pragma unroll
      for (int k = 0; k < Q; ++k) {
        const uint64_t j = base | loc[k0 + k];
        const double2 o = first ? cz() : os[j];
        os[j] = make_double2(fma(scale, r[k].x, o.x), fma(scale, r[k].y, o.y));
      }
    }
    __syncthreads();
  }
}

// Pauli coefficients of a 2x2 matrix M = sum_P a_P P with a_P = tr(P M)/2 (P in I,X,Y,Z).
void pauli_decompose(const double* m, cdd a[4]) {
  const cdd m00(m[0], m[1]), m10(m[2], m[3]), m01(m[4], m[5]), m11(m[6], m[7]);
  a[0] = (m00 + m11) / 2.0;                  // I
  a[1] = (m01 + m10) / 2.0;                  // X: tr(XM) = m10 + m01
  a[2] = (cdd(0, 1) * m01 - cdd(0, 1) * m10) / 2.0;  // Y: tr(YM) = -i m10 + i m01
  a[3] = (m00 - m11) / 2.0;                  // Z
}

}  // namespace

int pauli_compile(mb_observable o, const mb_term* terms, size_t nterms) {
  std::map<std::pair<uint64_t, uint64_t>, cdd> acc;  // (x, z) -> coefficient incl. i^{#Y}
  for (size_t t = 0; t < nterms; ++t) {
    const mb_term& tm = terms[t];
    struct Item {
      uint64_t x, z;
      int ny;
      cdd c;
    };
    std::vector<Item> cur{{0, 0, 0, cdd(tm.coeff[0], tm.coeff[1])}};
    for (int j = 0; j < tm.nsites; ++j) {
      cdd a[4];
      pauli_decompose(tm.ops + 8 * j, a);
      const uint64_t bit = uint64_t(1) << tm.sites[j];
      std::vector<Item> nxt;
      for (const Item& it : cur)
        for (int p = 0; p < 4; ++p) {
          if (a[p] == cdd(0, 0)) continue;
          Item n2 = it;
          n2.c *= a[p];
          if (p == 1 || p == 2) n2.x |= bit;
          if (p == 2 || p == 3) n2.z |= bit;
          if (p == 2) n2.ny += 1;
          nxt.push_back(n2);
        }
      cur.swap(nxt);
    }
    for (const Item& it : cur) {
      static const cdd ipow[4] = {cdd(1, 0), cdd(0, 1), cdd(-1, 0), cdd(0, -1)};
      acc[{it.x, it.z}] += it.c * ipow[it.ny & 3];
    }
  }
  auto* pd = new PauliData();
  uint64_t prev = ~uint64_t(0);
  for (auto& kv : acc) {
    if (kv.second == cdd(0, 0)) continue;
    const uint64_t x = kv.first.first;
    if (x != prev) {
      pd->groups.push_back({x, {int(pd->strings.size()), 0}});
      prev = x;
    }
    pd->strings.push_back(PString{kv.first.second, make_double2(kv.second.real(), kv.second.imag())});
    pd->groups.back().second.second += 1;
  }
  o->pauli = pd;
  o->pauli_ok = true;
  return MB_OK;
}

void pauli_free(mb_observable o) {
  if (!o->pauli) return;
  for (PauliProgram* p : o->pauli->programs) {
    dev_free(p->d_groups);
    dev_free(p->d_strings);
    dev_free(p->d_tables);
    dev_free(p->d_coef);
    for (void* f : p->jit)
      if (f) jit_release(f);
    delete p;
  }
  delete o->pauli;
  o->pauli = nullptr;
}

thread_local bool t_pauli_compile = true;

// Specialised kernels (mbk_pauli) for the passes of a program from MB_PAULI_JIT_MIN_BITS qubits
// (default 14; MB_PAULI_JIT=0 disables them). A pass whose per-thread factors would take too
// many registers, or whose kernel does not compile, keeps the interpreter kernel, and so do
// programs built on a thread that may not compile (the serving loop: a request's observable
// is often new, and neither NVRTC nor the source generation belongs on its path).
static void pauli_specialise(PauliData* pd, PauliProgram* P, const std::vector<PGroup>& hg,
                             const std::vector<std::vector<int>>& pass_groups) {
  P->jit.assign(P->passes.size(), nullptr);
  const int min_bits = getenv("MB_PAULI_JIT_MIN_BITS") ? atoi(getenv("MB_PAULI_JIT_MIN_BITS")) : 14;
  const char* e = getenv("MB_PAULI_JIT");
  if ((e && atoi(e) == 0) || P->n < min_bits || !t_pauli_compile || !jit_available() || pd->strings.empty()) return;
  std::vector<std::string> src;
  std::vector<size_t> which;
  // Passes of 2^12-amplitude tiles (from 24 qubits) keep the interpreter unless
  // MB_PAULI_JIT_WIDE=1: their per-thread factors fill the registers, and with them on, a
  // 24-qubit gradient alternating with a density-matrix gradient ran 2-3.5x slower per step
  // than either alone (cause not identified).
  const char* wide = getenv("MB_PAULI_JIT_WIDE");
  const bool wide_ok = wide && atoi(wide) == 1;
  for (size_t i = 0; i < P->passes.size(); ++i) {
    const PPassArgs& pa = P->passes[i];
    if (pa.ngroups == 0 || (pa.nr > 5 && !wide_ok)) continue;
    PauliJitPass jp;
    // 3 CTAs per SM for 2^10-amplitude tiles (0.84 against 0.90 ms for XXZ on 50 samples of 20
    // qubits at 2), 2 for 2^12 ones, whose per-thread factors need more registers
    jp.ctas = pa.nr <= 5 ? 3 : 2;
    if (const char* e = getenv("MB_PAULI_CTAS")) jp.ctas = atoi(e);
    jp.n = pa.n;
    jp.nr = pa.nr;
    for (int r = 0; r < kPRMax; ++r) jp.reg[r] = r < pa.nr ? pa.reg[r] : 0;
    for (size_t k = 0; k < pass_groups[i].size(); ++k) {
      const int g = pass_groups[i][k];
      const PGroup& G = hg[pa.g0 + k];
      PauliJitGroup jg;
      jg.x = G.x;
      jg.xl = G.xl;
      jg.herm = G.herm;
      jg.hb = G.hb;
      const int s0 = pd->groups[g].second.first, ns = pd->groups[g].second.second;
      for (int s = s0; s < s0 + ns; ++s) jg.strings.push_back(PauliJitString{s, pd->strings[s].z, pd->strings[s].c.y == 0.0});
      jp.groups.push_back(jg);
    }
    std::string code = jit_pauli_source(jp, 48);
    if (code.empty()) continue;
    src.push_back(std::move(code));
    which.push_back(i);
  }
  if (src.empty()) return;
  std::vector<double2> coef;
  for (const PString& ps : pd->strings) coef.push_back(ps.c);
  if (dev_alloc((void**)&P->d_coef, sizeof(double2) * coef.size()) != MB_OK) return;
  if (cudaMemcpyAsync(P->d_coef, coef.data(), sizeof(double2) * coef.size(), cudaMemcpyHostToDevice, g_ctx.stream) !=
          cudaSuccess ||
      cudaStreamSynchronize(g_ctx.stream) != cudaSuccess)
    return;
  std::vector<CUfunction> fns;
  std::string err;
  if (jit_prepare(src, fns, &err, 0.0) != MB_OK) {
    if (getenv("MB_JIT_VERBOSE")) fprintf(stderr, "mossb200: Pauli passes interpreted: %s\n", err.c_str());
    return;
  }
  // a kernel that spills to local memory keeps the interpreter pass
  for (size_t k = 0; k < which.size(); ++k) {
    if (!fns[k] || jit_local_bytes((void*)fns[k]) != 0) continue;
    P->jit[which[k]] = (void*)fns[k];
    jit_retain((void*)fns[k]);
  }
}

// Pass plan for an n-qubit state, or nullptr when the fused form does not apply (fewer than
// 10 qubits, or a group flips more register bits than a tile holds: 7 from 24 qubits, else 5).
// Each pass takes the groups whose flip bits fit its local bits; per group the strings are
// ordered constant, per-amplitude, tabulated, and the tabulated ones (strings inside the
// tile) are summed here over the tile's local indices.
static int pauli_program(mb_observable o, int n, PauliProgram** out) {
  *out = nullptr;
  PauliData* pd = o->pauli;
  if (!pd || n < 10) return MB_OK;
  // large tiles from MB_PAULI_WIDE_BITS qubits (default 24: fewer passes pay off for long
  // passes; at 20-22 qubits the smaller tiles measured faster on XXZ batches); tables for groups
  // with at least MB_PAULI_TABLE_MIN strings inside the tile (default 1: a table lookup is
  // cheaper than one per-amplitude parity)
  static const int wide_from = getenv("MB_PAULI_WIDE_BITS") ? atoi(getenv("MB_PAULI_WIDE_BITS")) : 24;
  static const int table_min = getenv("MB_PAULI_TABLE_MIN") ? atoi(getenv("MB_PAULI_TABLE_MIN")) : kPTableMin;
  const int nr = n >= wide_from && n >= 12 ? 7 : 5, local = 5 + nr;
  for (PauliProgram* p : pd->programs)
    if (p->n == n) {
      *out = p;
      return MB_OK;
    }
  std::vector<int> rem;
  for (size_t g = 0; g < pd->groups.size(); ++g) {
    const uint64_t hi = pd->groups[g].first & ~uint64_t(31);
    if (__builtin_popcountll(hi) > nr || (pd->groups[g].first >> n) != 0) return MB_OK;
    const int s0 = pd->groups[g].second.first, ns = pd->groups[g].second.second;
    for (int s = s0; s < s0 + ns; ++s)
      if ((pd->strings[s].z >> n) != 0) return MB_OK;
    rem.push_back(int(g));
  }
  std::unique_ptr<PauliProgram> P(new PauliProgram());
  P->n = n;
  P->nr = nr;
  std::vector<PGroup> hg;
  std::vector<PString> hs;
  std::vector<double2> ht;
  std::vector<std::vector<int>> pass_groups;  // the observable's groups each pass evaluates
  while (!rem.empty() || P->passes.empty()) {
    uint64_t regm = 0;
    for (int g : rem) {
      const uint64_t hi = pd->groups[g].first & ~uint64_t(31);
      if (__builtin_popcountll(regm | hi) <= nr) regm |= hi;
    }
    for (int q = n - 1; q >= 5 && __builtin_popcountll(regm) < nr; --q) regm |= uint64_t(1) << q;
    PPassArgs pa{};
    pa.n = n;
    pa.nr = nr;
    int k = 0;
    for (int q = 5; q < n; ++q)
      if ((regm >> q) & 1) pa.reg[k++] = q;
    const uint64_t localm = uint64_t(31) | regm;
    pa.g0 = int(hg.size());
    std::vector<int> left, took;
    for (int g : rem) {
      const uint64_t x = pd->groups[g].first;
      if ((x & ~localm) != 0 || int(hg.size()) - pa.g0 >= kPMaxGroups) {
        left.push_back(g);
        continue;
      }
      PGroup G{};
      G.x = x;
      G.xl = int(x & 31);
      for (int r = 0; r < nr; ++r)
        if ((x >> pa.reg[r]) & 1) G.xl |= 1 << (5 + r);
      const int s0 = pd->groups[g].second.first, ns = pd->groups[g].second.second;
      std::vector<PString> kc, st, tb;
      G.herm = 1;
      G.hb = G.xl ? 31 - __builtin_clz(unsigned(G.xl)) : 0;
      for (int s = s0; s < s0 + ns; ++s) {
        const PString& ps = pd->strings[s];
        // coefficient without i^{#Y} (#Y = |x & z|) real: c * (-i)^{#Y} has no imaginary part
        const int ny = __builtin_popcountll(x & ps.z) & 3;
        if ((ny & 1) ? ps.c.x != 0.0 : ps.c.y != 0.0) G.herm = 0;
        const uint64_t zl = ps.z & localm, zh = ps.z & ~localm;
        (zl == 0 ? kc : (zh == 0 ? tb : st)).push_back(ps);
      }
      // strings inside the tile go to the table unless there are fewer than table_min
      if (int(tb.size()) < table_min) {
        st.insert(st.end(), tb.begin(), tb.end());
        tb.clear();
      }
      G.k0 = int(hs.size());
      G.nk = int(kc.size());
      hs.insert(hs.end(), kc.begin(), kc.end());
      G.v0 = int(hs.size());
      G.nv = int(st.size());
      hs.insert(hs.end(), st.begin(), st.end());
      G.tab = -1;
      if (!tb.empty()) {
        // sum over the strings inside the local bits, for every local index l
        G.tab = int(ht.size());
        for (int l = 0; l < (1 << local); ++l) {
          const uint64_t k_idx = local_bits(l, pa.reg, nr) ^ x;
          double2 f = cz();
          for (const PString& ps : tb) {
            const bool odd = __builtin_popcountll(k_idx & ps.z) & 1;
            f.x += odd ? -ps.c.x : ps.c.x;
            f.y += odd ? -ps.c.y : ps.c.y;
          }
          ht.push_back(f);
        }
      }
      hg.push_back(G);
      took.push_back(g);
    }
    pass_groups.push_back(took);
    pa.ngroups = int(hg.size()) - pa.g0;
    pa.tiles_per_sample = int64_t(1) << (n - local);
    P->passes.push_back(pa);
    rem.swap(left);
    if (pd->groups.empty()) break;
  }
  int rc;
  if (!hg.empty()) {
    if ((rc = dev_alloc((void**)&P->d_groups, sizeof(PGroup) * hg.size()))) return rc;
    MB_CHECK_CUDA(cudaMemcpyAsync(P->d_groups, hg.data(), sizeof(PGroup) * hg.size(), cudaMemcpyHostToDevice, g_ctx.stream));
  }
  if (!hs.empty()) {
    if ((rc = dev_alloc((void**)&P->d_strings, sizeof(PString) * hs.size()))) return rc;
    MB_CHECK_CUDA(cudaMemcpyAsync(P->d_strings, hs.data(), sizeof(PString) * hs.size(), cudaMemcpyHostToDevice,
                                  g_ctx.stream));
  }
  if (!ht.empty()) {
    if ((rc = dev_alloc((void**)&P->d_tables, sizeof(double2) * ht.size()))) return rc;
    MB_CHECK_CUDA(cudaMemcpyAsync(P->d_tables, ht.data(), sizeof(double2) * ht.size(), cudaMemcpyHostToDevice,
                                  g_ctx.stream));
  }
  MB_CHECK_CUDA(cudaStreamSynchronize(g_ctx.stream));
  for (PPassArgs& pa : P->passes) {
    pa.groups = P->d_groups;
    pa.strings = P->d_strings;
    pa.tables = P->d_tables;
  }
  pauli_specialise(pd, P.get(), hg, pass_groups);
  *out = P.get();
  pd->programs.push_back(P.release());
  return MB_OK;
}

void pauli_allow_compile(bool on) { t_pauli_compile = on; }

bool pauli_usable(mb_observable o, mb_state s) {
  PauliProgram* p = nullptr;
  if (pauli_program(o, s->n, &p) != MB_OK) return false;
  return p != nullptr;
}

int expect_pauli(mb_observable o, mb_state s, double2* out) {
  if (!out) out = g_ctx.results;
  PauliProgram* P = nullptr;
  if (g_ctx.capturing) {
    for (PauliProgram* q : o->pauli->programs)
      if (q->n == s->n) P = q;
    if (!P && s->n >= 10) {
      set_error("record the expectation once before capturing it (its pass plan is built lazily)");
      return MB_EUNSUPPORTED;
    }
  } else {
    int rc = pauli_program(o, s->n, &P);
    if (rc) return rc;
  }
  if (!P) return expect_keys(o, s, out);
  cudaStream_t st = g_ctx.stream;
  MB_CHECK_CUDA(cudaMemsetAsync(out, 0, sizeof(double2) * s->batch, st));
  for (size_t i = 0; i < P->passes.size(); ++i) {
    const PPassArgs& pa = P->passes[i];
    if (pa.ngroups == 0) continue;
    int64_t per = std::max<int64_t>(1, std::min<int64_t>(int64_t(g_ctx.sm_count) * 8 / s->batch + 1,
                                                      g_ctx.partials_cap / (s->batch + 1) - 1));
    const int G = int(std::min<int64_t>(pa.tiles_per_sample, per));
    if (int64_t(G) * s->batch > g_ctx.partials_cap || s->batch > g_ctx.ncounters) {
      set_error("reduction workspace too small for %d samples", s->batch);
      return MB_EUNSUPPORTED;
    }
    const size_t shm = size_t(16) << (5 + pa.nr);
    if (i < P->jit.size() && P->jit[i]) {
      ProfScope ps("mbk_pauli", 16.0 * double(s->elems) * s->batch, st);
      if (int rc = jit_launch_pauli((CUfunction)P->jit[i], s->d, P->d_coef, pa.tiles_per_sample, g_ctx.partials,
                                    g_ctx.counters, out, G, s->batch, pauli_jit_shm(pa.nr), st))
        return rc;
      MB_LAUNCHED();
      continue;
    }
    ProfScope ps("k_pauli_pass", 16.0 * double(s->elems) * s->batch, st);
    auto launch = [&](auto kern) {
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(shm));
      kern<<<dim3(G, s->batch), kPThreads, shm, st>>>(s->d, pa, g_ctx.partials, g_ctx.counters, out);
    };
    pa.nr == 7 ? launch(k_pauli_pass<7>) : launch(k_pauli_pass<5>);
    MB_LAUNCHED();
  }
  return MB_OK;
}

// out = scale * H in for pure states (the adjoint seed 2H psi); false when the fused form
// does not apply to this register size (the caller then uses the per-key kernels).
int pauli_apply(mb_observable o, const double2* in, double2* out, int n, int nsamples, double scale, bool* done) {
  *done = false;
  PauliProgram* P = nullptr;
  int rc = pauli_program(o, n, &P);
  if (rc || !P) return rc;
  cudaStream_t st = g_ctx.stream;
  bool first = true;
  for (const PPassArgs& pa : P->passes) {
    if (pa.ngroups == 0) continue;
    const int G = int(std::min<int64_t>(pa.tiles_per_sample, int64_t(g_ctx.sm_count) * 16));
    ProfScope ps("k_pauli_apply", (first ? 32.0 : 48.0) * double(int64_t(1) << n) * nsamples, st);
    const size_t shm = size_t(16) << (5 + pa.nr);
    auto launch = [&](auto kern) {
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(shm));
      kern<<<dim3(G, nsamples), kPThreads, shm, st>>>(in, out, pa, scale, first ? 1 : 0);
    };
    pa.nr == 7 ? launch(k_pauli_apply<7>) : launch(k_pauli_apply<5>);
    MB_LAUNCHED();
    first = false;
  }
  if (first) MB_CHECK_CUDA(cudaMemsetAsync(out, 0, sizeof(double2) * (size_t(1) << n) * nsamples, st));
  *done = true;
  return MB_OK;
}

}  // namespace mb
