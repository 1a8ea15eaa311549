// Host-only harness for tests/test_jit_sources.py: generates specialised-kernel sources (Pauli
// expectation passes, a persistent uneven launch, a tile pass, a dual-state reverse pass with a
// gradient accumulator) from hand-built pass descriptions, compiles
// each with NVRTC for sm_100a (no GPU needed) and prints one JSON line per source with the
// compile status, registers and spill bytes reported by ptxas.
#include <dlfcn.h>

#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <regex>
#include <string>
#include <vector>

#include "jit.h"

namespace mb {
void set_error(const char* f, ...) {
  va_list a;
  va_start(a, f);
  vfprintf(stderr, f, a);
  va_end(a);
  fputc('\n', stderr);
}
}  // namespace mb

using namespace mb;

typedef int (*create_t)(void**, const char*, const char*, int, const char* const*, const char* const*);
typedef int (*compile_t)(void*, int, const char* const*);
typedef int (*logsz_t)(void*, size_t*);
typedef int (*log_t)(void*, char*);
typedef int (*destroy_t)(void**);

static void compile_and_report(const char* name, const std::string& src) {
  static void* h = nullptr;
  if (!h) h = dlopen("libnvrtc.so.12", RTLD_NOW);
  if (!h) h = dlopen("libnvrtc.so", RTLD_NOW);
  if (!h) {
    printf("{\"name\": \"%s\", \"bytes\": %zu, \"rc\": -1, \"error\": \"no NVRTC\"}\n", name, src.size());
    return;
  }
  auto create = (create_t)dlsym(h, "nvrtcCreateProgram");
  auto compile = (compile_t)dlsym(h, "nvrtcCompileProgram");
  auto logsz = (logsz_t)dlsym(h, "nvrtcGetProgramLogSize");
  auto getlog = (log_t)dlsym(h, "nvrtcGetProgramLog");
  auto destroy = (destroy_t)dlsym(h, "nvrtcDestroyProgram");
  void* prog = nullptr;
  create(&prog, src.c_str(), "mbk.cu", 0, nullptr, nullptr);
  const char* opts[] = {"--gpu-architecture=sm_100a", "-std=c++17", "--fmad=true", "-default-device",
                        "--ptxas-options=-v"};
  const int rc = compile(prog, 5, opts);
  size_t ls = 0;
  logsz(prog, &ls);
  std::string log(ls, '\0');
  if (ls) getlog(prog, &log[0]);
  destroy(&prog);
  int regs = -1, spill = -1;
  std::smatch m;
  if (std::regex_search(log, m, std::regex("Used ([0-9]+) registers"))) regs = std::stoi(m[1]);
  if (std::regex_search(log, m, std::regex("([0-9]+) bytes spill stores"))) spill = std::stoi(m[1]);
  printf("{\"name\": \"%s\", \"bytes\": %zu, \"rc\": %d, \"regs\": %d, \"spill\": %d}\n", name, src.size(), rc, regs,
         spill);
  if (rc != 0) fprintf(stderr, "%s\n", log.substr(0, 3000).c_str());
}

// Nearest-neighbour Hamiltonian on n qubits as one pass of 2^10-amplitude tiles with register
// bits regs[0..4]: the diagonal group (Z Z on every pair) and, for every pair inside the
// tile's bits, a flip group (X X, and Y Y when xxz).
static PauliJitPass nn_pass(int n, const int* regs, bool xxz) {
  PauliJitPass p{};
  p.n = n;
  p.nr = 5;
  p.ctas = 3;
  uint64_t localm = 31;
  for (int r = 0; r < 5; ++r) {
    p.reg[r] = regs[r];
    localm |= uint64_t(1) << regs[r];
  }
  int s = 0;
  PauliJitGroup diag{0, 0, 1, 0, {}};
  for (int i = 0; i + 1 < n; ++i) diag.strings.push_back({s++, (uint64_t(1) << i) | (uint64_t(1) << (i + 1)), true});
  p.groups.push_back(diag);
  for (int i = 0; i + 1 < n; ++i) {
    const uint64_t x = xxz ? (uint64_t(1) << i) | (uint64_t(1) << (i + 1)) : uint64_t(1) << i;
    if ((x & ~localm) != 0) continue;
    PauliJitGroup g{x, 0, 1, 0, {}};
    int xl = int(x & 31);
    for (int r = 0; r < 5; ++r)
      if ((x >> regs[r]) & 1) xl |= 1 << (5 + r);
    g.xl = xl;
    g.hb = 31 - __builtin_clz(unsigned(xl));
    g.strings.push_back({s++, 0, true});
    if (xxz) g.strings.push_back({s++, x, true});
    p.groups.push_back(g);
  }
  return p;
}

static MOp mop(int type, int r0, int r1, std::vector<int> sel, uint32_t active, int param, std::vector<int> off) {
  MOp m{};
  m.type = int16_t(type);
  m.r0 = int16_t(r0);
  m.r1 = int16_t(r1);
  m.nsel = int16_t(sel.size());
  for (size_t i = 0; i < sel.size(); ++i) m.sel[i] = int16_t(sel[i]);
  m.active = active;
  m.param = int16_t(param);
  for (size_t i = 0; i < off.size(); ++i) m.off[i] = off[i];
  return m;
}

static StageDesc stage(int op0, int nops, std::vector<int> reg, std::vector<int> tid) {
  StageDesc s{};
  s.op0 = op0;
  s.nops = nops;
  s.nreg = int(reg.size());
  for (size_t i = 0; i < reg.size(); ++i) s.reg[i] = reg[i];
  s.ntid = int(tid.size());
  for (size_t i = 0; i < tid.size(); ++i) s.tid[i] = tid[i];
  return s;
}

// A tile pass over local bits 0..t-1 with register width 3: per-sample and fixed 2x2 gates, a
// sign flip under a thread-bit condition, a diagonal factor and a per-sample derived product.
static Pass tile_pass(int t) {
  Pass p;
  p.kind = PASS_TILE;
  p.t = t;
  for (int q = 0; q < t; ++q) p.bits.push_back(q);
  p.mops.push_back(mop(MOP_U1, 0, 0, {}, 0, 1, {0, 1, 2, 3}));
  p.mops.push_back(mop(MOP_CPHASE, 0, 1, {0, 3}, 0, 0, {}));
  p.mops.push_back(mop(MOP_U1, 1, 0, {}, 0, 0, {4, 5, 6, 7}));
  p.mops.push_back(mop(MOP_DIAG, 0, 0, {4}, 0x2, 0, {8, 9}));
  p.mops.push_back(mop(MOP_U1, 2, 0, {}, 0, 1, {kXtabFlag | 0, kXtabFlag | 1, kXtabFlag | 2, kXtabFlag | 3}));
  std::vector<int> rest;
  for (int q = 3; q < t; ++q) rest.push_back(q);
  p.stages.push_back(stage(0, 2, {0, 1, 2}, rest));
  std::vector<int> tid2 = {0, 1, 2};
  for (int q = 6; q < t; ++q) tid2.push_back(q);
  p.stages.push_back(stage(2, 3, {3, 4, 5}, tid2));
  return p;
}

int main() {
  const int low[5] = {5, 6, 7, 8, 9}, high[5] = {9, 10, 11, 12, 13};
  compile_and_report("pauli_xxz_n20_bits5_9", jit_pauli_source(nn_pass(20, low, true), 48));
  compile_and_report("pauli_xxz_n20_bits9_13", jit_pauli_source(nn_pass(20, high, true), 48));
  compile_and_report("pauli_tfim_n22_bits5_9", jit_pauli_source(nn_pass(22, low, false), 48));
  compile_and_report("pauli_xxz_n22_bits5_9", jit_pauli_source(nn_pass(22, low, true), 48));
  const Pass p10 = tile_pass(10), p8 = tile_pass(8);
  std::vector<UnevenJitPass> passes = {{&p10, 14, true, 4}, {&p10, 14, false, 4}, {&p8, 8, true, 1}};
  int threads = 0;
  size_t shm = 0;
  const std::string src = jit_uneven_source(passes, 3, 4, &threads, &shm);
  compile_and_report("uneven_n14_n8", src);
  printf("{\"name\": \"uneven_launch\", \"threads\": %d, \"shm\": %zu}\n", threads, shm);
  // a tile pass and a dual-state reverse pass (with a rotation-generator gradient) of a
  // 14-qubit state: TMA boxes over bits 0..9 of a two-dimensional amplitude tensor
  Pass pt = tile_pass(10);
  pt.geom.ndims = 2;
  pt.geom.start[0] = 0;
  pt.geom.bits[0] = 10;
  pt.geom.boxb[0] = 10;
  pt.geom.start[1] = 10;
  pt.geom.bits[1] = 4;
  pt.geom.boxb[1] = 0;
  compile_and_report("tile_n14", jit_tile_source(pt, 3, 14, false, 4));
  Pass pa = pt;
  pa.mops.push_back(mop(MOP_GRADP, 0, 2, {}, 0, 0, {}));  // closes stage 1 (ops 2..5)
  pa.stages[1].nops += 1;
  pa.grad_slots = {0};
  compile_and_report("adjoint_n14", jit_adjoint_source(pa, 3, 14, true, 3));
  return 0;
}
