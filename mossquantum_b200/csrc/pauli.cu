// K4: fused Pauli-string expectation <psi|H|psi> (bit masks, phases and warp shuffles).
//
// The reference evaluates one dense local matrix per site key, one state pass per key
// (src/observables/expectation.jl:12-33, backends/cpu/expectations/threaded.jl). Here every
// term is decomposed into Pauli strings P = i^{#Y} X^x Z^z with a complex coefficient, and
// the strings are grouped by their flip mask x. For amplitude index j,
//   <psi|P|psi> = sum_j conj(psi_j) * i^{#Y} (-1)^{|(j^x)&z|} psi_{j^x}.
// One pass gives each warp 32 consecutive low indices (lanes = bits 0..4) and each thread
// 2^R amplitudes on R higher "register" bits. A group whose flip mask lies in those bits
// finds its partner amplitude in the thread's registers (mirrored in shared memory for the
// runtime flip) and a warp shuffle across lanes, so one read of the state evaluates every
// such group; the diagonal group (x = 0: all Z/ZZ terms) needs no partner. Groups with flip
// bits elsewhere run in further passes with other register bits; TFIM on n qubits takes
// ceil((n-5)/5) passes instead of 2n-1.
#include <algorithm>
#include <cmath>
#include <complex>
#include <map>
#include <memory>
#include <vector>

#include "internal.h"

namespace mb {

typedef std::complex<double> cdd;
constexpr int kPR = 5;  // register bits per thread
constexpr int kPThreads = 64;   // 64 x 32 mirrored amplitudes = 32 KiB of shared memory

struct PString {
  uint64_t z;
  double2 c;  // coefficient including i^{#Y}
};

struct PGroup {
  uint64_t x;  // flip mask (global bits)
  int xlow;    // flip bits among lanes (bits 0..4)
  int xreg;    // flip bits among the register bits (register index space)
  int s0, ns;  // strings [s0, s0 + ns)
};

struct PPassArgs {
  int n;
  int reg[kPR];
  int g0, ngroups;
  const PGroup* groups;
  const PString* strings;
  int64_t threads_per_sample;
};

struct PauliProgram {
  int n = -1;
  std::vector<PPassArgs> passes;
  PGroup* d_groups = nullptr;
  PString* d_strings = nullptr;
};

struct PauliData {
  std::vector<PString> strings;  // grouped by flip mask
  std::vector<std::pair<uint64_t, std::pair<int, int>>> groups;  // x -> [s0, ns)
  std::vector<PauliProgram*> programs;
};

namespace {

__device__ __forceinline__ double2 warp_sum2(double2 x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    x.x += __shfl_down_sync(0xffffffffu, x.x, o);
    x.y += __shfl_down_sync(0xffffffffu, x.y, o);
  }
  return x;
}

__global__ void __launch_bounds__(kPThreads) k_pauli_pass(const double2* __restrict__ v, const PPassArgs a,
                                                         double2* partials, unsigned* counters, double2* out) {
  __shared__ double2 mirror[1 << kPR][kPThreads];
  __shared__ double2 wp[kPThreads / 32];
  __shared__ bool last;
  const int b = blockIdx.y, G = gridDim.x;
  const double2* vs = v + (int64_t(b) << a.n);
  int reg[kPR];
#pragma unroll
  for (int k = 0; k < kPR; ++k) reg[k] = a.reg[k];
  double2 acc = cz();
  // Every lane of a warp iterates the same number of times (the per-sample thread count is
  // a multiple of 32), so the shuffles below always see a full warp.
  for (int64_t t0 = int64_t(blockIdx.x) * blockDim.x; t0 < a.threads_per_sample; t0 += int64_t(G) * blockDim.x) {
    const int64_t t = t0 + threadIdx.x;
    if (t >= a.threads_per_sample) break;  // whole warps leave together (count is a multiple of 32)
    uint64_t base = uint64_t(t);
#pragma unroll
    for (int k = 0; k < kPR; ++k) {
      const int p = reg[k];
      base = ((base >> p) << (p + 1)) | (base & ((uint64_t(1) << p) - 1));
    }
    double2 amp[1 << kPR];
#pragma unroll
    for (int j = 0; j < (1 << kPR); ++j) {
      uint64_t o = 0;
#pragma unroll
      for (int k = 0; k < kPR; ++k)
        if ((j >> k) & 1) o |= uint64_t(1) << reg[k];
      amp[j] = vs[base | o];
      mirror[j][threadIdx.x] = amp[j];
    }
    __syncwarp();
    for (int gi = 0; gi < a.ngroups; ++gi) {
      const PGroup g = a.groups[a.g0 + gi];
#pragma unroll
      for (int j = 0; j < (1 << kPR); ++j) {
        uint64_t o = 0;
#pragma unroll
        for (int k = 0; k < kPR; ++k)
          if ((j >> k) & 1) o |= uint64_t(1) << reg[k];
        const uint64_t k_idx = (base | o) ^ g.x;  // index of the partner amplitude
        double2 p = g.xreg ? mirror[j ^ g.xreg][threadIdx.x] : amp[j];
        if (g.xlow) {
          p.x = __shfl_xor_sync(0xffffffffu, p.x, g.xlow);
          p.y = __shfl_xor_sync(0xffffffffu, p.y, g.xlow);
        }
        double2 f = cz();
        for (int s = 0; s < g.ns; ++s) {
          const PString ps = a.strings[g.s0 + s];
          const bool odd = __popcll(k_idx & ps.z) & 1;
          f.x += odd ? -ps.c.x : ps.c.x;
          f.y += odd ? -ps.c.y : ps.c.y;
        }
        // conj(psi_j) * psi_{j^x} * f
        const double2 cp = make_double2(amp[j].x * p.x + amp[j].y * p.y, amp[j].x * p.y - amp[j].y * p.x);
        acc = cfma(f, cp, acc);
      }
    }
    __syncwarp();
  }
  acc = warp_sum2(acc);
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
// Same pass structure as k_pauli_pass; each pass adds the groups it holds.
__global__ void __launch_bounds__(kPThreads) k_pauli_apply(const double2* __restrict__ v, double2* __restrict__ out,
                                                          const PPassArgs a, double scale, int first) {
  __shared__ double2 mirror[1 << kPR][kPThreads];
  const int b = blockIdx.y, G = gridDim.x;
  const double2* vs = v + (int64_t(b) << a.n);
  double2* os = out + (int64_t(b) << a.n);
  int reg[kPR];
#pragma unroll
  for (int k = 0; k < kPR; ++k) reg[k] = a.reg[k];
  for (int64_t t0 = int64_t(blockIdx.x) * blockDim.x; t0 < a.threads_per_sample; t0 += int64_t(G) * blockDim.x) {
    const int64_t t = t0 + threadIdx.x;
    if (t >= a.threads_per_sample) break;
    uint64_t base = uint64_t(t);
#pragma unroll
    for (int k = 0; k < kPR; ++k) {
      const int p = reg[k];
      base = ((base >> p) << (p + 1)) | (base & ((uint64_t(1) << p) - 1));
    }
#pragma unroll
    for (int j = 0; j < (1 << kPR); ++j) {
      uint64_t o = 0;
#pragma unroll
      for (int k = 0; k < kPR; ++k)
        if ((j >> k) & 1) o |= uint64_t(1) << reg[k];
      mirror[j][threadIdx.x] = vs[base | o];
    }
#pragma unroll
    for (int j = 0; j < (1 << kPR); ++j) {
      uint64_t o = 0;
#pragma unroll
      for (int k = 0; k < kPR; ++k)
        if ((j >> k) & 1) o |= uint64_t(1) << reg[k];
      double2 r = first ? cz() : os[base | o];
      for (int gi = 0; gi < a.ngroups; ++gi) {
        const PGroup g = a.groups[a.g0 + gi];
        double2 p = mirror[j ^ g.xreg][threadIdx.x];
        if (g.xlow) {
          p.x = __shfl_xor_sync(0xffffffffu, p.x, g.xlow);
          p.y = __shfl_xor_sync(0xffffffffu, p.y, g.xlow);
        }
        const uint64_t k_idx = (base | o) ^ g.x;
        double2 f = cz();
        for (int s = 0; s < g.ns; ++s) {
          const PString ps = a.strings[g.s0 + s];
          const bool odd = __popcll(k_idx & ps.z) & 1;
          f.x += odd ? -ps.c.x : ps.c.x;
          f.y += odd ? -ps.c.y : ps.c.y;
        }
        r = cfma(cscale(f, scale), p, r);
      }
      os[base | o] = r;
    }
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
    delete p;
  }
  delete o->pauli;
  o->pauli = nullptr;
}

// Pass plan for an n-qubit state, or nullptr when the fused form does not apply (fewer
// than 5 + R qubits, or a group flips more than R bits above the lane bits).
static int pauli_program(mb_observable o, int n, PauliProgram** out) {
  *out = nullptr;
  PauliData* pd = o->pauli;
  if (!pd || n < 5 + kPR) return MB_OK;
  for (PauliProgram* p : pd->programs)
    if (p->n == n) {
      *out = p;
      return MB_OK;
    }
  std::vector<int> rem;
  for (size_t g = 0; g < pd->groups.size(); ++g) {
    const uint64_t hi = pd->groups[g].first & ~uint64_t(31);
    if (__builtin_popcountll(hi) > kPR) return MB_OK;
    rem.push_back(int(g));
  }
  std::unique_ptr<PauliProgram> P(new PauliProgram());
  P->n = n;
  std::vector<PGroup> hg;
  while (!rem.empty() || P->passes.empty()) {
    uint64_t regm = 0;
    for (int g : rem) {
      const uint64_t hi = pd->groups[g].first & ~uint64_t(31);
      if (__builtin_popcountll(regm | hi) <= kPR) regm |= hi;
    }
    for (int q = n - 1; q >= 5 && __builtin_popcountll(regm) < kPR; --q) regm |= uint64_t(1) << q;
    PPassArgs pa{};
    pa.n = n;
    int k = 0;
    for (int q = 5; q < n; ++q)
      if ((regm >> q) & 1) pa.reg[k++] = q;
    pa.g0 = int(hg.size());
    std::vector<int> left;
    for (int g : rem) {
      const uint64_t x = pd->groups[g].first;
      if ((x & ~uint64_t(31) & ~regm) != 0) {
        left.push_back(g);
        continue;
      }
      PGroup G{};
      G.x = x;
      G.xlow = int(x & 31);
      for (int r = 0; r < kPR; ++r)
        if ((x >> pa.reg[r]) & 1) G.xreg |= 1 << r;
      G.s0 = pd->groups[g].second.first;
      G.ns = pd->groups[g].second.second;
      hg.push_back(G);
    }
    pa.ngroups = int(hg.size()) - pa.g0;
    pa.threads_per_sample = int64_t(1) << (n - kPR);
    P->passes.push_back(pa);
    rem.swap(left);
    if (pd->groups.empty()) break;
  }
  int rc;
  if (!hg.empty()) {
    if ((rc = dev_alloc((void**)&P->d_groups, sizeof(PGroup) * hg.size()))) return rc;
    MB_CHECK_CUDA(cudaMemcpyAsync(P->d_groups, hg.data(), sizeof(PGroup) * hg.size(), cudaMemcpyHostToDevice, g_ctx.stream));
  }
  if (!pd->strings.empty()) {
    if ((rc = dev_alloc((void**)&P->d_strings, sizeof(PString) * pd->strings.size()))) return rc;
    MB_CHECK_CUDA(cudaMemcpyAsync(P->d_strings, pd->strings.data(), sizeof(PString) * pd->strings.size(),
                                  cudaMemcpyHostToDevice, g_ctx.stream));
  }
  MB_CHECK_CUDA(cudaStreamSynchronize(g_ctx.stream));
  for (PPassArgs& pa : P->passes) {
    pa.groups = P->d_groups;
    pa.strings = P->d_strings;
  }
  *out = P.get();
  pd->programs.push_back(P.release());
  return MB_OK;
}

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
    if (!P && s->n >= 5 + kPR) {
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
  for (const PPassArgs& pa : P->passes) {
    if (pa.ngroups == 0) continue;
    const int64_t blocks = (pa.threads_per_sample + kPThreads - 1) / kPThreads;
    int64_t per = std::max<int64_t>(1, std::min<int64_t>(int64_t(g_ctx.sm_count) * 8 / s->batch + 1,
                                                      g_ctx.partials_cap / (s->batch + 1) - 1));
    const int G = int(std::min<int64_t>(blocks, per));
    if (int64_t(G) * s->batch > g_ctx.partials_cap || s->batch > g_ctx.ncounters) {
      set_error("reduction workspace too small for %d samples", s->batch);
      return MB_EUNSUPPORTED;
    }
    ProfScope ps("k_pauli_pass", 16.0 * double(s->elems) * s->batch, st);
    k_pauli_pass<<<dim3(G, s->batch), kPThreads, 0, st>>>(s->d, pa, g_ctx.partials, g_ctx.counters, out);
    MB_LAUNCHED();
  }
  return MB_OK;
}

}  // namespace mb

namespace mb {
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
    const int64_t blocks = (pa.threads_per_sample + kPThreads - 1) / kPThreads;
    const int G = int(std::min<int64_t>(blocks, int64_t(g_ctx.sm_count) * 16));
    ProfScope ps("k_pauli_apply", (first ? 32.0 : 48.0) * double(int64_t(1) << n) * nsamples, st);
    k_pauli_apply<<<dim3(G, nsamples), kPThreads, 0, st>>>(in, out, pa, scale, first ? 1 : 0);
    MB_LAUNCHED();
    first = false;
  }
  if (first) MB_CHECK_CUDA(cudaMemsetAsync(out, 0, sizeof(double2) * (size_t(1) << n) * nsamples, st));
  *done = true;
  return MB_OK;
}
}  // namespace mb
