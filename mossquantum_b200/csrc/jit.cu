// Runtime-specialised pass kernels (NVRTC).
//
// The interpreter kernels (k_tile_pass / k_reg_pass) decode micro-ops at run time. For large
// states this module instead generates one straight-line kernel per pass structure: the
// register offsets, swizzled shared-memory slots, matrix-table offsets and control patterns
// are compile-time constants, a controlled-X on register bits becomes a renaming of
// variables (no instructions), and a CZ a handful of sign flips. Matrix values stay in the
// circuit's table, so circuits that differ only in angles share one kernel. Kernels are
// compiled with NVRTC for sm_100a, cached by their source text, and launched through the
// driver API on the library stream.
#include <cuda.h>
#include <dlfcn.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "jit.h"

namespace mb {
namespace {

// ---- NVRTC (dlopen'ed) -----------------------------------------------------------------------
typedef int nvrtcResult_t;
typedef struct _nvrtcProgram* nvrtcProgram_t;
struct Nvrtc {
  void* h = nullptr;
  nvrtcResult_t (*create)(nvrtcProgram_t*, const char*, const char*, int, const char* const*, const char* const*);
  nvrtcResult_t (*compile)(nvrtcProgram_t, int, const char* const*);
  nvrtcResult_t (*log_size)(nvrtcProgram_t, size_t*);
  nvrtcResult_t (*log)(nvrtcProgram_t, char*);
  nvrtcResult_t (*cubin_size)(nvrtcProgram_t, size_t*);
  nvrtcResult_t (*cubin)(nvrtcProgram_t, char*);
  nvrtcResult_t (*destroy)(nvrtcProgram_t*);
  bool ok = false;
};

Nvrtc& nvrtc() {
  static Nvrtc n;
  static bool tried = false;
  if (tried) return n;
  tried = true;
  const char* paths[] = {"libnvrtc.so.12", "/usr/local/cuda/lib64/libnvrtc.so.12", "libnvrtc.so"};
  for (const char* p : paths) {
    n.h = dlopen(p, RTLD_NOW | RTLD_LOCAL);
    if (n.h) break;
  }
  if (!n.h) return n;
  n.create = (decltype(n.create))dlsym(n.h, "nvrtcCreateProgram");
  n.compile = (decltype(n.compile))dlsym(n.h, "nvrtcCompileProgram");
  n.log_size = (decltype(n.log_size))dlsym(n.h, "nvrtcGetProgramLogSize");
  n.log = (decltype(n.log))dlsym(n.h, "nvrtcGetProgramLog");
  n.cubin_size = (decltype(n.cubin_size))dlsym(n.h, "nvrtcGetCUBINSize");
  n.cubin = (decltype(n.cubin))dlsym(n.h, "nvrtcGetCUBIN");
  n.destroy = (decltype(n.destroy))dlsym(n.h, "nvrtcDestroyProgram");
  n.ok = n.create && n.compile && n.log_size && n.log && n.cubin_size && n.cubin && n.destroy;
  return n;
}

// ---- driver API (through the runtime's entry-point query) -----------------------------------
struct Drv {
  CUresult (*load)(CUmodule*, const void*) = nullptr;
  CUresult (*getfn)(CUfunction*, CUmodule, const char*) = nullptr;
  CUresult (*launch)(CUfunction, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned, CUstream,
                     void**, void**) = nullptr;
  CUresult (*setattr)(CUfunction, CUfunction_attribute, int) = nullptr;
  CUresult (*getattr)(int*, CUfunction_attribute, CUfunction) = nullptr;
  CUresult (*unload)(CUmodule) = nullptr;
  bool ok = false;
};

Drv& drv() {
  static Drv d;
  static bool tried = false;
  if (tried) return d;
  tried = true;
  cudaDriverEntryPointQueryResult q;
  void* p = nullptr;
  if (cudaGetDriverEntryPoint("cuModuleLoadData", &p, cudaEnableDefault, &q) == cudaSuccess && p) d.load = (decltype(d.load))p;
  if (cudaGetDriverEntryPoint("cuModuleGetFunction", &p, cudaEnableDefault, &q) == cudaSuccess && p) d.getfn = (decltype(d.getfn))p;
  if (cudaGetDriverEntryPoint("cuLaunchKernel", &p, cudaEnableDefault, &q) == cudaSuccess && p) d.launch = (decltype(d.launch))p;
  if (cudaGetDriverEntryPoint("cuFuncSetAttribute", &p, cudaEnableDefault, &q) == cudaSuccess && p) d.setattr = (decltype(d.setattr))p;
  if (cudaGetDriverEntryPoint("cuModuleUnload", &p, cudaEnableDefault, &q) == cudaSuccess && p) d.unload = (decltype(d.unload))p;
  if (cudaGetDriverEntryPoint("cuFuncGetAttribute", &p, cudaEnableDefault, &q) == cudaSuccess && p) d.getattr = (decltype(d.getattr))p;
  d.ok = d.load && d.getfn && d.launch && d.setattr;
  return d;
}

// Compiled kernels by source text. Schedules that use a kernel hold a reference
// (jit_retain / jit_release); jit_trim unloads the least recently used unreferenced modules
// while more than MB_JIT_CACHE_MAX (default 1024) are loaded, so a long-running process that
// meets ever new circuit shapes keeps a bounded set of modules.
struct CacheEnt {
  CUmodule mod = nullptr;
  CUfunction fn = nullptr;
  int refs = 0;
  uint64_t last = 0;
};
std::mutex g_jit_mu;
std::map<std::string, CacheEnt> g_cache;
std::map<CUfunction, std::string> g_by_fn;
uint64_t g_tick = 0;
double g_compile_s = 0.0;     // cumulative NVRTC compile + module load time
uint64_t g_compiles = 0;

const char* kPrelude = R"PRE(
typedef unsigned long long u64;
typedef unsigned int u32;
struct __align__(64) TMap { u64 v[16]; };
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cfma(double2 a, double2 b, double2 c) {
  return make_double2(fma(a.x, b.x, fma(-a.y, b.y, c.x)), fma(a.x, b.y, fma(a.y, b.x, c.y)));
}
__device__ __forceinline__ double2 ld(const double2* p) { return __ldg(p); }
__device__ __forceinline__ double2 ldc(const double2* p) { double2 x = __ldg(p); return make_double2(x.x, -x.y); }
__device__ __forceinline__ double2 neg(double2 a) { return make_double2(-a.x, -a.y); }
__device__ __forceinline__ double2 cneg(double2 a, u64 s) {
  return make_double2(__longlong_as_double(__double_as_longlong(a.x) ^ (long long)s),
                      __longlong_as_double(__double_as_longlong(a.y) ^ (long long)s));
}
__device__ __forceinline__ double2 cj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ u32 swz(u32 i) { return i ^ ((i >> 3) & 7u); }
__device__ __forceinline__ u32 sa(const void* p) { return (u32)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(u64* b) { asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(sa(b)) : "memory"); }
__device__ __forceinline__ void mbar_tx(u64* b, u32 n) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(sa(b)), "r"(n) : "memory");
}
__device__ __forceinline__ bool mbar_wait(u64* b, u32 ph) {
  for (u32 it = 0; it < (1u << 26); ++it) {
    u32 done;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
                 : "=r"(done) : "r"(sa(b)), "r"(ph) : "memory");
    if (done) return true;
  }
  return false;
}
)PRE";

std::string tma_ld(int nd) {
  std::ostringstream o;
  o << "asm volatile(\"cp.async.bulk.tensor." << nd
    << "d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {";
  for (int d = 0; d < nd; ++d) o << (d ? ", " : "") << "%" << (2 + d);
  o << "}], [%" << (2 + nd) << "];\" :: \"r\"(sa(DST)), \"l\"((u64)&tmap)";
  for (int d = 0; d < nd; ++d) o << ", \"r\"(c" << d << ")";
  o << ", \"r\"(sa(BAR)) : \"memory\");";
  return o.str();
}

std::string tma_st(int nd) {
  std::ostringstream o;
  o << "asm volatile(\"cp.async.bulk.tensor." << nd << "d.global.shared::cta.tile.bulk_group [%0, {";
  for (int d = 0; d < nd; ++d) o << (d ? ", " : "") << "%" << (2 + d);
  o << "}], [%1];\" :: \"l\"((u64)&tmap), \"r\"(sa(SRC))";
  for (int d = 0; d < nd; ++d) o << ", \"r\"(c" << d << ")";
  o << " : \"memory\"); asm volatile(\"cp.async.bulk.commit_group;\" ::: \"memory\");";
  return o.str();
}

// Shared-memory staging key of matrix element e of a micro-op: its table offset, with bit 30 set
// for a per-sample derived entry (those live in their own row region, so their offsets can
// coincide with fixed derived ones).
constexpr int32_t kXrowKey = 1 << 30;
inline int smat_key(const MOp& m, int e) {
  return m.off[e] | ((m.param && (m.off[e] & kXtabFlag)) ? kXrowKey : 0);
}

// Generates the body of one register stage. Variables a0..a{2^R-1} hold the amplitudes; nm
// maps logical register index j to the variable currently holding it (controlled-X on
// register bits only permutes nm).
struct StageGen {
  int R;
  const int* reg;      // pass-local bit of register bit k
  std::ostringstream& o;
  bool lb64;           // pass-local index is a 64-bit global index (register sweep)
  std::vector<int> nm;
  std::string pre = "a";  // variable prefix
  const std::map<int, int>* smap = nullptr;  // table offset -> slot of the pass's shared-memory copy
  const std::map<int, int>* pmap = nullptr;  // per-sample entry -> slot of the tile's shared copy (spar)
  int pkey = 0;        // added to the smap key of per-sample entries (copies holding both kinds)

  // Selector classification: register bit k (>= 0), or -1 with a runtime expression.
  int regbit(int sel) const {
    if (sel >= 64) return -1;
    for (int k = 0; k < R; ++k)
      if (reg[k] == sel) return k;
    return -1;
  }
  std::string rt(int sel) const {
    std::ostringstream e;
    if (sel >= 64) e << "(u32)((gb >> " << (sel - 64) << ") & 1ull)";
    else e << "(u32)((lb >> " << sel << ") & 1" << (lb64 ? "ull" : "u") << ")";
    return e.str();
  }
  // Splits selectors into a compile-time register mask and a runtime condition string.
  void split(const MOp& m, int& need, std::string& cond) const {
    need = 0;
    cond.clear();
    for (int c = 0; c < m.nsel; ++c) {
      const int k = regbit(m.sel[c]);
      if (k >= 0) need |= 1 << k;
      else cond += (cond.empty() ? "" : " & ") + rt(m.sel[c]);
    }
  }
  std::string v(int j) const { return pre + std::to_string(nm[j]); }
  std::string ldm(const MOp& m, int e) const {
    if (smap) {
      auto it = smap->find(smat_key(m, e) | (m.param ? pkey : 0));
      if (it != smap->end()) {
        const std::string x = "smat[" + std::to_string(it->second) + "]";
        return m.conj ? "cj(" + x + ")" : x;
      }
    }
    if (pmap && m.param) {
      auto it = pmap->find(smat_key(m, e));
      if (it != pmap->end()) {
        const std::string x = "spar[" + std::to_string(it->second) + "]";
        return m.conj ? "cj(" + x + ")" : x;
      }
    }
    if (m.off[e] & kXtabFlag)
      return std::string(m.conj ? "ldc" : "ld") + "(" + (m.param ? "xb" : "xtab") + " + " +
             std::to_string(m.off[e] & ~kXtabFlag) + ")";
    return std::string(m.conj ? "ldc" : "ld") + "(" + (m.param ? "tb" : "tab") + " + " + std::to_string(m.off[e]) + ")";
  }

  void emit(const MOp& m) {
    const int A = 1 << R;
    switch (m.type) {
      case MOP_U1: {
        const int b = 1 << m.r0;
        o << "{ const double2 m00 = " << ldm(m, 0) << ", m10 = " << ldm(m, 1) << ", m01 = " << ldm(m, 2)
          << ", m11 = " << ldm(m, 3) << ";\n";
        for (int j = 0; j < A; ++j)
          if (!(j & b))
            o << "  { const double2 ux = " << v(j) << ", uy = " << v(j | b) << "; " << v(j)
              << " = cfma(m01, uy, cmul(m00, ux)); " << v(j | b) << " = cfma(m11, uy, cmul(m10, ux)); }\n";
        o << "}\n";
        break;
      }
      case MOP_RROT: {
        const int b = 1 << m.r0;
        o << "{ const double ra = (" << ldm(m, 0) << ").x, rc = (" << ldm(m, 1) << ").x, rb = (" << ldm(m, 2)
          << ").x, rd = (" << ldm(m, 3) << ").x;\n";
        for (int j = 0; j < A; ++j)
          if (!(j & b))
            o << "  { const double2 ux = " << v(j) << ", uy = " << v(j | b) << "; " << v(j)
              << " = make_double2(fma(rb, uy.x, ra * ux.x), fma(rb, uy.y, ra * ux.y)); " << v(j | b)
              << " = make_double2(fma(rd, uy.x, rc * ux.x), fma(rd, uy.y, rc * ux.y)); }\n";
        o << "}\n";
        break;
      }
      case MOP_IROT: {
        // [[a, i bi], [i ci, d]]
        const int b = 1 << m.r0;
        o << "{ const double ra = (" << ldm(m, 0) << ").x, ci = (" << ldm(m, 1) << ").y, bi = (" << ldm(m, 2)
          << ").y, rd = (" << ldm(m, 3) << ").x;\n";
        for (int j = 0; j < A; ++j)
          if (!(j & b))
            o << "  { const double2 ux = " << v(j) << ", uy = " << v(j | b) << "; " << v(j)
              << " = make_double2(fma(-bi, uy.y, ra * ux.x), fma(bi, uy.x, ra * ux.y)); " << v(j | b)
              << " = make_double2(fma(-ci, ux.y, rd * uy.x), fma(ci, ux.x, rd * uy.y)); }\n";
        o << "}\n";
        break;
      }
      case MOP_LIFT: {
        // three shears: x += mt*y; y += s*x; x += mt*y (per component)
        const int b = 1 << m.r0;
        o << "{ const double2 ts = " << ldm(m, 0) << ";\n";
        for (int j = 0; j < A; ++j)
          if (!(j & b)) {
            const std::string x = v(j), y = v(j | b);
            o << "  " << x << ".x = fma(ts.x, " << y << ".x, " << x << ".x); " << x << ".y = fma(ts.x, " << y << ".y, " << x
              << ".y); " << y << ".x = fma(ts.y, " << x << ".x, " << y << ".x); " << y << ".y = fma(ts.y, " << x << ".y, "
              << y << ".y); " << x << ".x = fma(ts.x, " << y << ".x, " << x << ".x); " << x << ".y = fma(ts.x, " << y
              << ".y, " << x << ".y);\n";
          }
        o << "}\n";
        break;
      }
      case MOP_CTRL: {
        const int b = 1 << m.r0;
        int need;
        std::string cond;
        split(m, need, cond);
        o << "{ const double2 m00 = " << ldm(m, 0) << ", m10 = " << ldm(m, 1) << ", m01 = " << ldm(m, 2)
          << ", m11 = " << ldm(m, 3) << ";\n";
        if (!cond.empty()) o << " if (" << cond << ") {\n";
        for (int j = 0; j < A; ++j)
          if (!(j & b) && (j & need) == need)
            o << "  { const double2 ux = " << v(j) << ", uy = " << v(j | b) << "; " << v(j)
              << " = cfma(m01, uy, cmul(m00, ux)); " << v(j | b) << " = cfma(m11, uy, cmul(m10, ux)); }\n";
        if (!cond.empty()) o << " }\n";
        o << "}\n";
        break;
      }
      case MOP_CTRLX: {
        const int b = 1 << m.r0;
        int need;
        std::string cond;
        split(m, need, cond);
        if (cond.empty()) {
          for (int j = 0; j < A; ++j)
            if (!(j & b) && (j & need) == need) std::swap(nm[j], nm[j | b]);
        } else {
          o << "{ const bool pr = (" << cond << ") != 0u;\n";
          for (int j = 0; j < A; ++j)
            if (!(j & b) && (j & need) == need)
              o << "  { const double2 ux = " << v(j) << ", uy = " << v(j | b) << "; " << v(j) << " = pr ? uy : ux; "
                << v(j | b) << " = pr ? ux : uy; }\n";
          o << "}\n";
        }
        break;
      }
      case MOP_CPHASE: {
        int need;
        std::string cond;
        split(m, need, cond);
        if (m.r1 && !cond.empty()) {
          // a sign flip under a thread or tile condition: flip the sign bits without a branch
          // (no divergence inside a warp, one basic block for the scheduler)
          o << "{ const u64 sg = (u64)(" << cond << ") << 63;\n";
          for (int j = 0; j < A; ++j)
            if ((j & need) == need) o << "  " << v(j) << " = cneg(" << v(j) << ", sg);\n";
          o << "}\n";
          break;
        }
        o << "{ ";
        if (!m.r1) o << "const double2 f = " << ldm(m, 0) << "; ";
        if (!cond.empty()) o << "if (" << cond << ") {";
        o << "\n";
        for (int j = 0; j < A; ++j)
          if ((j & need) == need) o << "  " << v(j) << " = " << (m.r1 ? "neg(" + v(j) + ")" : "cmul(f, " + v(j) + ")") << ";\n";
        if (!cond.empty()) o << " }";
        o << "}\n";
        break;
      }
      case MOP_CHAN: {
        const int b0 = 1 << m.r0, b1 = 1 << m.r1;
        o << "{ const double ca = (" << ldm(m, 0) << ").x, cb = (" << ldm(m, 1) << ").x, cc = (" << ldm(m, 2)
          << ").x, cd = (" << ldm(m, 3) << ").x, ce = (" << ldm(m, 4) << ").x, cf = (" << ldm(m, 5) << ").x;\n";
        for (int j = 0; j < A; ++j)
          if (!(j & b0) && !(j & b1)) {
            const std::string x0 = v(j), x1 = v(j | b0), x2 = v(j | b1), x3 = v(j | b0 | b1);
            o << "  { const double2 p0 = " << x0 << ", p3 = " << x3 << "; " << x0
              << " = make_double2(fma(ca, p0.x, cb * p3.x), fma(ca, p0.y, cb * p3.y)); " << x3
              << " = make_double2(fma(ce, p0.x, cf * p3.x), fma(ce, p0.y, cf * p3.y)); " << x1 << " = make_double2(cc * "
              << x1 << ".x, cc * " << x1 << ".y); " << x2 << " = make_double2(cd * " << x2 << ".x, cd * " << x2
              << ".y); }\n";
          }
        o << "}\n";
        break;
      }
      case MOP_U2: {
        const int b0 = 1 << m.r0, b1 = 1 << m.r1;
        o << "{ double2 u[16];\n";
        for (int e = 0; e < 16; ++e) o << " u[" << e << "] = " << ldm(m, e) << ";";
        o << "\n";
        for (int j = 0; j < A; ++j)
          if (!(j & b0) && !(j & b1)) {
            const int i[4] = {j, j | b0, j | b1, j | b0 | b1};
            o << "  { const double2 x0 = " << v(i[0]) << ", x1 = " << v(i[1]) << ", x2 = " << v(i[2]) << ", x3 = " << v(i[3])
              << ";\n";
            for (int r = 0; r < 4; ++r)
              o << "    " << v(i[r]) << " = cfma(u[" << (12 + r) << "], x3, cfma(u[" << (8 + r) << "], x2, cfma(u["
                << (4 + r) << "], x1, cmul(u[" << r << "], x0))));\n";
            o << "  }\n";
          }
        o << "}\n";
        break;
      }
      case MOP_DIAG: {
        // Factor index = register part (known here) | runtime part (thread or tile bits). For
        // every register part the factor is chosen among the runtime combinations with selects,
        // so nothing is indexed at run time (no local-memory array).
        int rk[4];
        std::vector<int> rtsel;
        for (int c = 0; c < m.nsel; ++c) {
          rk[c] = regbit(m.sel[c]);
          if (rk[c] < 0) rtsel.push_back(c);
        }
        o << "{ ";
        for (int e = 0; e < (1 << m.nsel); ++e)
          if ((m.active >> e) & 1) o << "const double2 F" << e << " = " << ldm(m, e) << "; ";
        for (size_t r = 0; r < rtsel.size(); ++r) o << "const bool r" << r << " = " << rt(m.sel[rtsel[r]]) << " != 0u; ";
        o << "\n";
        int ctmask = 0;
        for (int c = 0; c < m.nsel; ++c)
          if (rk[c] >= 0) ctmask |= 1 << c;
        // factor expression for register part ct: a select tree over the runtime bits
        std::function<std::string(int, size_t)> fexpr = [&](int idx, size_t r) -> std::string {
          if (r == rtsel.size())
            return ((m.active >> idx) & 1) ? "F" + std::to_string(idx) : std::string("make_double2(1.0, 0.0)");
          const std::string a = fexpr(idx, r + 1), b = fexpr(idx | (1 << rtsel[r]), r + 1);
          return a == b ? a : "(r" + std::to_string(r) + " ? " + b + " : " + a + ")";
        };
        std::map<int, std::string> gname;
        for (int j = 0; j < A; ++j) {
          int ct = 0;
          for (int c = 0; c < m.nsel; ++c)
            if (rk[c] >= 0 && ((j >> rk[c]) & 1)) ct |= 1 << c;
          // factors of 1 for every runtime combination: nothing to do
          bool any = false;
          for (int rc = 0; rc < (1 << m.nsel); ++rc)
            if ((rc & ctmask) == ct && ((m.active >> rc) & 1)) any = true;
          if (!any) continue;
          if (!gname.count(ct)) {
            gname[ct] = "G" + std::to_string(ct);
            o << "  const double2 " << gname[ct] << " = " << fexpr(ct, 0) << ";\n";
          }
          o << "  " << v(j) << " = cmul(" << gname[ct] << ", " << v(j) << ");\n";
        }
        o << "}\n";
        break;
      }
    }
  }
};

std::string reg_off_const(int j, int R, const int* reg) {
  unsigned long long c = 0;
  for (int k = 0; k < R; ++k)
    if ((j >> k) & 1) c |= 1ull << reg[k];
  return std::to_string(c) + "ull";
}

// Entry point of a generated source: mbk_tile (tile pass), mbk_reg (strided sweep), mbk_adj
// (adjoint dual-state pass), mbk_uneven (persistent launch over several register sizes) or
// mbk_pauli (Pauli-string expectation pass).
const char* kernel_name(const std::string& src) {
  if (src.find(" mbk_uneven(") != std::string::npos) return "mbk_uneven";
  if (src.find(" mbk_pauli(") != std::string::npos) return "mbk_pauli";
  if (src.find(" mbk_adj(") != std::string::npos) return "mbk_adj";
  if (src.find(" mbk_reg(") != std::string::npos) return "mbk_reg";
  return "mbk_tile";
}

// Compiles (or fetches) a kernel; returns nullptr on any failure.
CUfunction compile_kernel(const std::string& src, std::string* err) {
  {
    std::lock_guard<std::mutex> lk(g_jit_mu);
    auto it = g_cache.find(src);
    if (it != g_cache.end()) {
      it->second.last = ++g_tick;
      return it->second.fn;
    }
  }
  Nvrtc& n = nvrtc();
  Drv& d = drv();
  if (!n.ok || !d.ok) {
    *err = "NVRTC or driver entry points unavailable";
    return nullptr;
  }
  nvrtcProgram_t prog;
  if (n.create(&prog, src.c_str(), "mbk.cu", 0, nullptr, nullptr) != 0) {
    *err = "nvrtcCreateProgram failed";
    return nullptr;
  }
  const char* opts[] = {"--gpu-architecture=sm_100a", "-std=c++17", "--fmad=true", "-default-device"};
  const auto t0 = std::chrono::steady_clock::now();
  const int rc = n.compile(prog, 4, opts);
  if (getenv("MB_JIT_VERBOSE")) {
    const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    fprintf(stderr, "mossb200: compiled a %zu-byte pass in %.2f s\n", src.size(), sec);
  }
  if (const char* dir = getenv("MB_JIT_DUMP")) {
    // Development aid: every compiled source and its compile time.
    const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    const size_t h = std::hash<std::string>()(src);
    char path[512];
    snprintf(path, sizeof(path), "%s/mbk_%016zx.cu", dir, h);
    if (FILE* f = fopen(path, "w")) {
      fwrite(src.data(), 1, src.size(), f);
      fclose(f);
    }
    snprintf(path, sizeof(path), "%s/compile_times.txt", dir);
    std::lock_guard<std::mutex> lk(g_jit_mu);
    if (FILE* f = fopen(path, "a")) {
      fprintf(f, "mbk_%016zx %.3f s %zu bytes rc=%d\n", h, sec, src.size(), rc);
      fclose(f);
    }
  }
  if (rc != 0) {
    size_t ls = 0;
    n.log_size(prog, &ls);
    std::string log(ls, '\0');
    n.log(prog, &log[0]);
    *err = "NVRTC compile failed: " + log.substr(0, 2000);
    n.destroy(&prog);
    return nullptr;
  }
  size_t cs = 0;
  n.cubin_size(prog, &cs);
  std::vector<char> cubin(cs);
  n.cubin(prog, cubin.data());
  n.destroy(&prog);
  CUmodule mod;
  CUfunction fn;
  if (d.load(&mod, cubin.data()) != CUDA_SUCCESS || d.getfn(&fn, mod, kernel_name(src)) != CUDA_SUCCESS) {
    *err = "module load failed";
    return nullptr;
  }
  std::lock_guard<std::mutex> lk(g_jit_mu);
  auto it = g_cache.find(src);
  if (it != g_cache.end()) {  // another thread compiled the same source meanwhile
    if (d.unload) d.unload(mod);
    it->second.last = ++g_tick;
    return it->second.fn;
  }
  CacheEnt& e = g_cache[src];
  e.mod = mod;
  e.fn = fn;
  e.last = ++g_tick;
  g_by_fn[fn] = src;
  g_compile_s += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  ++g_compiles;
  return fn;
}

}  // namespace

bool jit_available() { return nvrtc().ok && drv().ok; }

int jit_local_bytes(void* fn) {
  Drv& d = drv();
  int v = -1;
  if (!fn || !d.getattr || d.getattr(&v, CU_FUNC_ATTRIBUTE_LOCAL_SIZE_BYTES, (CUfunction)fn) != CUDA_SUCCESS) return -1;
  return v;
}

void jit_retain(void* fn) {
  std::lock_guard<std::mutex> lk(g_jit_mu);
  auto it = g_by_fn.find((CUfunction)fn);
  if (it != g_by_fn.end()) ++g_cache[it->second].refs;
}

void jit_release(void* fn) {
  std::lock_guard<std::mutex> lk(g_jit_mu);
  auto it = g_by_fn.find((CUfunction)fn);
  if (it != g_by_fn.end()) {
    CacheEnt& e = g_cache[it->second];
    if (e.refs > 0) --e.refs;
  }
}

void jit_trim() {
  size_t cap = 1024;
  if (const char* e = getenv("MB_JIT_CACHE_MAX")) cap = size_t(std::max(16, atoi(e)));
  Drv& d = drv();
  std::lock_guard<std::mutex> lk(g_jit_mu);
  bool synced = false;
  while (g_cache.size() > cap && d.unload) {
    auto victim = g_cache.end();
    for (auto it = g_cache.begin(); it != g_cache.end(); ++it)
      if (it->second.refs == 0 && (victim == g_cache.end() || it->second.last < victim->second.last)) victim = it;
    if (victim == g_cache.end()) break;  // everything loaded is in use
    if (!synced) {
      // a released schedule's kernels may still be running: finish all work before unloading
      cudaDeviceSynchronize();
      synced = true;
    }
    d.unload(victim->second.mod);
    g_by_fn.erase(victim->second.fn);
    g_cache.erase(victim);
  }
}

void jit_stats(double* compile_ms, uint64_t* compiles, size_t* modules) {
  std::lock_guard<std::mutex> lk(g_jit_mu);
  if (compile_ms) *compile_ms = g_compile_s * 1e3;
  if (compiles) *compiles = g_compiles;
  if (modules) *modules = g_cache.size();
}

// Matrix elements of a pass that are the same for every sample (fixed gates and channels): the
// kernel copies them from the table into shared memory once per CTA, so the gate loops read
// them with uniform shared-memory loads instead of global loads. At most 2048 entries (32 KB).
struct SharedMats {
  std::map<int, int> slot;
  std::vector<int> offs;
};

// with_params: also stage the per-sample (parametric) elements and derivative generators;
// valid for single-sample schedules, where every thread reads sample 0's row.
static SharedMats shared_mats(const Pass& p, bool with_params) {
  SharedMats sm;
  const MOp* cur = nullptr;
  auto add = [&](int e) {
    const int key = smat_key(*cur, e);
    if (sm.slot.count(key)) return;
    sm.slot[key] = int(sm.offs.size());
    sm.offs.push_back(key);
  };
  for (const MOp& m : p.mops) {
    if (m.param && !with_params) continue;
    cur = &m;
    switch (m.type) {
      case MOP_U1: case MOP_CTRL: case MOP_RROT: case MOP_IROT: for (int e = 0; e < 4; ++e) add(e); break;
      case MOP_LIFT: add(0); break;
      case MOP_U2: for (int e = 0; e < 16; ++e) add(e); break;
      case MOP_CHAN: for (int e = 0; e < 6; ++e) add(e); break;
      case MOP_DIAG: for (int e = 0; e < (1 << m.nsel); ++e) if ((m.active >> e) & 1) add(e); break;
      case MOP_CPHASE: if (!m.r1) add(0); break;
      case MOP_GRAD: for (int e = 0; e < (m.nsel == 1 ? 4 : 16); ++e) add(e); break;
      default: break;
    }
  }
  if (sm.offs.size() > 2048) sm = SharedMats();
  return sm;
}

// Per-sample matrix elements of a multi-sample pass (parametric gates, fused per-sample
// products): every tile belongs to one sample, so the tile's elements are copied into shared
// memory once per tile and the stages read them from there. At most 1024 entries (16 KB).
static SharedMats per_sample_mats(const Pass& p) {
  SharedMats sm;
  const MOp* cur = nullptr;
  auto add = [&](int e) {
    const int key = smat_key(*cur, e);
    if (sm.slot.count(key)) return;
    sm.slot[key] = int(sm.offs.size());
    sm.offs.push_back(key);
  };
  for (const MOp& m : p.mops) {
    if (!m.param) continue;
    cur = &m;
    switch (m.type) {
      case MOP_U1: case MOP_CTRL: case MOP_RROT: case MOP_IROT: for (int e = 0; e < 4; ++e) add(e); break;
      case MOP_LIFT: add(0); break;
      case MOP_U2: for (int e = 0; e < 16; ++e) add(e); break;
      case MOP_DIAG: for (int e = 0; e < (1 << m.nsel); ++e) if ((m.active >> e) & 1) add(e); break;
      case MOP_CPHASE: if (!m.r1) add(0); break;
      default: break;
    }
  }
  if (sm.offs.size() > 1024) sm = SharedMats();
  return sm;
}

// File-scope table of the offsets and the in-kernel copy (run before the kernel's first barrier).
static std::string shared_mats_decl(const SharedMats& sm) {
  if (sm.offs.empty()) return "";
  std::ostringstream o;
  o << "__constant__ int k_moffs[" << sm.offs.size() << "] = {";
  for (size_t i = 0; i < sm.offs.size(); ++i) o << (i ? "," : "") << sm.offs[i];
  o << "};\n";
  return o.str();
}
static std::string shared_mats_fill(const SharedMats& sm) {
  if (sm.offs.empty()) return "";
  std::ostringstream o;
  o << "  __shared__ double2 smat[" << sm.offs.size() << "];\n  for (u32 i = threadIdx.x; i < " << sm.offs.size()
    << "u; i += blockDim.x) { const int mo = k_moffs[i]; smat[i] = (mo & " << kXrowKey << ") ? __ldg(xtabs + (mo & "
    << (kXtabFlag - 1) << ")) : (mo & " << kXtabFlag << ") ? __ldg(xtab + (mo & " << (kXtabFlag - 1)
    << ")) : __ldg(tab + mo); }\n";
  return o.str();
}

// Barrier after register stage i: none after the last (the proxy fence and the CTA barrier
// before the tile's store follow); __syncwarp when stage i+1 keeps the same warp-index bits
// (every warp then reads back only what it wrote); else a CTA barrier.
static const char* stage_sync(const Pass& p, size_t i) {
  if (i + 1 == p.stages.size()) return "";
  const StageDesc& a = p.stages[i];
  const StageDesc& b = p.stages[i + 1];
  bool same = a.ntid == b.ntid;
  for (int q = 5; same && q < a.ntid; ++q) same = a.tid[q] == b.tid[q];
  return same ? "      __syncwarp();\n" : "      __syncthreads();\n";
}

std::string jit_tile_source(const Pass& p, int R, int N, bool stage_params, int ctas) {
  std::ostringstream o;
  const int A = 1 << R;
  const int threads = 1 << (p.t - R);
  const TmaGeom& g = p.geom;
  const SharedMats smats = shared_mats(p, stage_params);
  const SharedMats pmats = stage_params ? SharedMats() : per_sample_mats(p);
  o << kPrelude << shared_mats_decl(smats);
  if (!pmats.offs.empty()) {
    o << "__constant__ int k_poffs[" << pmats.offs.size() << "] = {";
    for (size_t i = 0; i < pmats.offs.size(); ++i) o << (i ? "," : "") << pmats.offs[i];
    o << "};\n";
  }
  o << "extern \"C\" __global__ void __launch_bounds__(" << threads << ", " << std::max(1, ctas)
    << ") mbk_tile(const __grid_constant__ TMap tmap, "
    << "const double2* __restrict__ tab, const double2* __restrict__ xtab, const double2* __restrict__ xtabs, "
    << "long long xrow, long long tstride, long long tps, "
    << "long long ntiles, u32* err) {\n";
  o << "  extern __shared__ unsigned char smem_raw[];\n  __shared__ __align__(8) u64 bar[2];\n  __shared__ int s_abort;\n";
  o << shared_mats_fill(smats);
  if (!pmats.offs.empty()) o << "  __shared__ double2 spar[" << pmats.offs.size() << "];\n";
  o << "  double2* buf0 = (double2*)(((unsigned long long)smem_raw + 1023ull) & ~1023ull);\n";
  o << "  double2* bufs[2] = {buf0, buf0 + " << (1 << p.t) << "};\n";
  o << "  const u32 tx = threadIdx.x;\n";
  o << "  if (tx == 0) { mbar_init(&bar[0]); mbar_init(&bar[1]); asm volatile(\"fence.mbarrier_init.release.cluster;\" ::: \"memory\"); s_abort = 0; }\n";
  o << "  __syncthreads();\n";
  // geometry: base index with zeros at the tile bits, TMA coordinates
  auto geom = [&](const char* tile, const char* pre) {
    std::ostringstream e;
    e << "  const int " << pre << "b = (int)(" << tile << " / tps);\n";
    e << "  u64 " << pre << "gb = (u64)(" << tile << " - (long long)" << pre << "b * tps);\n";
    for (int q = 0; q < p.t; ++q) {
      const int bit = p.bits[q];
      e << "  " << pre << "gb = ((" << pre << "gb >> " << bit << ") << " << (bit + 1) << ") | (" << pre << "gb & "
        << ((1ull << bit) - 1) << "ull);\n";
    }
    for (int d = 0; d < g.ndims; ++d) {
      e << "  const int " << pre << "c" << d << " = ";
      if (g.start[d] < 0) e << pre << "b;\n";
      else if (d == 0) e << "(int)(2ull * (" << pre << "gb & " << ((1ull << g.bits[0]) - 1) << "ull));\n";
      else e << "(int)((" << pre << "gb >> " << g.start[d] << ") & " << ((1ull << g.bits[d]) - 1) << "ull);\n";
    }
    return e.str();
  };
  auto with_prefix = [&](std::string s, const char* pre) {
    // rename c{d} in the TMA strings to pre c{d}
    for (int d = 0; d < g.ndims; ++d) {
      const std::string from = "\"r\"(c" + std::to_string(d) + ")", to = std::string("\"r\"(") + pre + "c" + std::to_string(d) + ")";
      size_t pos;
      while ((pos = s.find(from)) != std::string::npos) s.replace(pos, from.size(), to);
    }
    return s;
  };
  std::string ld = tma_ld(g.ndims), st = tma_st(g.ndims);
  const unsigned bytes = 16u << p.t;
  o << "  u32 ph0 = 0, ph1 = 0;\n  long long tile = blockIdx.x;\n";
  o << "  if (tx == 0 && tile < ntiles) {\n" << geom("tile", "p_");
  {
    std::string s = with_prefix(ld, "p_");
    size_t pos;
    while ((pos = s.find("DST")) != std::string::npos) s.replace(pos, 3, "bufs[0]");
    while ((pos = s.find("BAR")) != std::string::npos) s.replace(pos, 3, "&bar[0]");
    o << "    mbar_tx(&bar[0], " << bytes << "u); " << s << "\n  }\n";
  }
  o << "  for (int it = 0; tile < ntiles; ++it, tile += gridDim.x) {\n";
  o << "    const int cur = it & 1;\n    const long long nxt = tile + gridDim.x;\n";
  o << "    if (tx == 0 && nxt < ntiles) {\n" << geom("nxt", "n_");
  {
    std::string s = with_prefix(ld, "n_");
    size_t pos;
    while ((pos = s.find("DST")) != std::string::npos) s.replace(pos, 3, "bufs[cur ^ 1]");
    while ((pos = s.find("BAR")) != std::string::npos) s.replace(pos, 3, "&bar[cur ^ 1]");
    o << "      asm volatile(\"cp.async.bulk.wait_group.read 0;\" ::: \"memory\");\n      mbar_tx(&bar[cur ^ 1], " << bytes
      << "u); " << s << "\n    }\n";
  }
  o << geom("tile", "");
  o << "    const double2* tb = tab + (long long)b * tstride;\n    (void)tb;\n";
  o << "    const double2* xb = xtabs + (long long)b * xrow;\n    (void)xb;\n";
  if (!pmats.offs.empty()) {
    // this tile's per-sample elements (the previous tile's stages ended with a barrier)
    o << "    for (u32 i = tx; i < " << pmats.offs.size() << "u; i += blockDim.x) { const int mo = k_poffs[i]; "
      << "spar[i] = (mo & " << kXrowKey << ") ? __ldg(xb + (mo & " << (kXtabFlag - 1) << ")) : __ldg(tb + mo); }\n";
  }
  o << "    double2* tl = bufs[cur];\n";
  o << "    if (!mbar_wait(&bar[cur], cur ? ph1 : ph0)) { atomicOr(err, 1u); s_abort = 1; }\n";
  o << "    if (cur) ph1 ^= 1u; else ph0 ^= 1u;\n    __syncthreads();\n    if (s_abort) break;\n";
  o << "    double2 ";
  for (int j = 0; j < A; ++j) o << (j ? ", " : "") << "a" << j;
  o << ";\n";
  for (size_t si = 0; si < p.stages.size(); ++si) {
    const StageDesc& sd = p.stages[si];
    o << "    {\n      const u32 lb = 0u";
    for (int q = 0; q < sd.ntid; ++q) o << " | (((tx >> " << q << ") & 1u) << " << sd.tid[q] << ")";
    o << ";\n";
    for (int j = 0; j < A; ++j) o << "      a" << j << " = tl[swz(lb | " << reg_off_const(j, R, sd.reg) << ")];\n";
    StageGen sg{R, sd.reg, o, false, std::vector<int>(A)};
    sg.smap = &smats.slot;
    if (!pmats.offs.empty()) sg.pmap = &pmats.slot;
    for (int j = 0; j < A; ++j) sg.nm[j] = j;
    for (int q = 0; q < sd.nops; ++q) sg.emit(p.mops[sd.op0 + q]);
    for (int j = 0; j < A; ++j) o << "      tl[swz(lb | " << reg_off_const(j, R, sd.reg) << ")] = " << sg.v(j) << ";\n";
    o << stage_sync(p, si) << "    }\n";
  }
  o << "    asm volatile(\"fence.proxy.async.shared::cta;\" ::: \"memory\");\n    __syncthreads();\n";
  {
    std::string s = st;
    size_t pos;
    while ((pos = s.find("SRC")) != std::string::npos) s.replace(pos, 3, "tl");
    o << "    if (tx == 0) { " << s << " }\n";
  }
  o << "  }\n  if (tx == 0) asm volatile(\"cp.async.bulk.wait_group 0;\" ::: \"memory\");\n}\n";
  (void)N;
  return o.str();
}

// Gradient accumulation of one MOP_GRAD op: thread sum of Re<y|D|delta> over its register
// amplitudes, reduced across the warp and added to the warp's shared-memory slot.
// Emits this thread's partial sum of one gradient micro-op into variable `name` (declared by
// the caller); the warp reduction of a stage's sums runs once, in emit_grad_reduce.
static void emit_grad(std::ostringstream& o, const MOp& m, const StageGen& gy, const StageGen& gd, int R,
                      const std::string& name) {
  const int A = 1 << R;
  const std::string tabn = m.param ? "tb" : "tab";
  // generator entries, conjugated for the column bits of a density matrix
  auto L = [&](int e) {
    if (gy.smap) {
      auto it = gy.smap->find(smat_key(m, e));
      if (it != gy.smap->end()) {
        const std::string x = "smat[" + std::to_string(it->second) + "]";
        return m.conj ? "cj(" + x + ")" : x;
      }
    }
    return std::string(m.conj ? "ldc" : "ld") + "(" + tabn + " + " + std::to_string(m.off[e]) + ")";
  };
  o << "{ double gs = 0.0;\n";
  if (m.type == MOP_GRADP) {
    // Constant generators: (i/2)X, (i/2)Y, (i/2)Z, diag(0, -i); Re<y|D|delta> per pair.
    const int b = 1 << m.r0;
    for (int j = 0; j < A; ++j)
      if (!(j & b)) {
        const std::string y0 = gy.v(j), y1 = gy.v(j | b), d0 = gd.v(j), d1 = gd.v(j | b);
        switch (m.r1) {
          case 1:
            o << "  gs = fma(" << y0 << ".y, " << d1 << ".x, gs); gs = fma(-" << y0 << ".x, " << d1 << ".y, gs); gs = fma("
              << y1 << ".y, " << d0 << ".x, gs); gs = fma(-" << y1 << ".x, " << d0 << ".y, gs);\n";
            break;
          case 2:
            o << "  gs = fma(" << y0 << ".x, " << d1 << ".x, gs); gs = fma(" << y0 << ".y, " << d1 << ".y, gs); gs = fma(-"
              << y1 << ".x, " << d0 << ".x, gs); gs = fma(-" << y1 << ".y, " << d0 << ".y, gs);\n";
            break;
          case 3:
            o << "  gs = fma(" << y0 << ".y, " << d0 << ".x, gs); gs = fma(-" << y0 << ".x, " << d0 << ".y, gs); gs = fma(-"
              << y1 << ".y, " << d1 << ".x, gs); gs = fma(" << y1 << ".x, " << d1 << ".y, gs);\n";
            break;
          default:
            o << "  gs = fma(" << y1 << ".x, " << d1 << ".y, gs); gs = fma(-" << y1 << ".y, " << d1 << ".x, gs);\n";
        }
      }
    // the 1/2 of the Pauli generators, and the sign of adjoint gates
    const double scale = (m.r1 == 4 ? 1.0 : 0.5) * (m.conj ? -1.0 : 1.0);
    o << "  gs *= " << (scale < 0 ? "-" : "") << (std::abs(scale) == 0.5 ? "0.5" : "1.0") << ";\n";
  } else if (m.nsel == 1) {
    const int b = 1 << m.r0;
    o << "  const double2 D00 = " << L(0) << ", D10 = " << L(1) << ", D01 = " << L(2) << ", D11 = " << L(3) << ";\n";
    for (int j = 0; j < A; ++j)
      if (!(j & b))
        o << "  { const double2 gq0 = " << gd.v(j) << ", gq1 = " << gd.v(j | b) << ", gl0 = " << gy.v(j) << ", gl1 = "
          << gy.v(j | b) << "; const double2 e0 = cfma(D01, gq1, cmul(D00, gq0)), e1 = cfma(D11, gq1, cmul(D10, gq0)); "
          << "gs += gl0.x * e0.x + gl0.y * e0.y + gl1.x * e1.x + gl1.y * e1.y; }\n";
  } else {
    const int b0 = 1 << m.r0, b1 = 1 << m.r1;
    o << "  double2 D[16];";
    for (int e = 0; e < 16; ++e) o << " D[" << e << "] = " << L(e) << ";";
    o << "\n";
    for (int j = 0; j < A; ++j)
      if (!(j & b0) && !(j & b1)) {
        const int i[4] = {j, j | b0, j | b1, j | b0 | b1};
        o << "  { const double2 gq0 = " << gd.v(i[0]) << ", gq1 = " << gd.v(i[1]) << ", gq2 = " << gd.v(i[2]) << ", gq3 = "
          << gd.v(i[3]) << ";\n";
        for (int r = 0; r < 4; ++r)
          o << "    { const double2 e = cfma(D[" << (12 + r) << "], gq3, cfma(D[" << (8 + r) << "], gq2, cfma(D[" << (4 + r)
            << "], gq1, cmul(D[" << r << "], gq0)))); const double2 gl = " << gy.v(i[r])
            << "; gs += gl.x * e.x + gl.y * e.y; }\n";
        o << "  }\n";
      }
  }
  o << "  " << name << " = gs;\n}\n";
}

// Sums k partial sums (consecutive accumulators acc0, acc0+1, ...) over the warp in one
// butterfly: at step s the lanes with lane bit s set keep the upper half of their values and
// send the lower half, so k values take (k - 1) + (5 - log2 k) shuffles instead of 5k. Lane L
// then holds the sum of value j = sum_s bit_s(L) * k / 2^(s+1); lanes below k add it to the
// warp's slot of accumulator acc0 + j.
static void emit_grad_reduce(std::ostringstream& o, const std::vector<std::string>& names, int acc0, int nw) {
  const int kreal = int(names.size());
  int k = 1, m = 0;
  while (k < kreal) k <<= 1, ++m;
  if (m > 5) return;  // callers chunk to 32
  o << "{ const u32 ln = tx & 31u;\n";
  for (int i = 0; i < k; ++i) o << "  double v" << i << " = " << (i < kreal ? names[i] : std::string("0.0")) << ";\n";
  int cur = k;
  for (int st = 0; st < m; ++st) {
    const int half = cur >> 1;
    o << "  { const bool up = (ln >> " << st << ") & 1u;\n";
    for (int i = 0; i < half; ++i)
      o << "    { const double keep = up ? v" << (i + half) << " : v" << i << ", send = up ? v" << i << " : v"
        << (i + half) << "; v" << i << " = keep + __shfl_xor_sync(0xffffffffu, send, " << (1 << st) << "); }\n";
    o << "  }\n";
    cur = half;
  }
  for (int st = m; st < 5; ++st) o << "  v0 += __shfl_xor_sync(0xffffffffu, v0, " << (1 << st) << ");\n";
  o << "  if (ln < " << k << "u) { u32 j = 0u;";
  for (int st = 0; st < m; ++st) o << " j += ((ln >> " << st << ") & 1u) * " << (k >> (st + 1)) << "u;";
  o << " if (j < " << kreal << "u) gw[(" << acc0 << "u + j) * " << nw << "u + (tx >> 5)] += v0; }\n}\n";
}

std::string jit_adjoint_source(const Pass& p, int R, int N, bool stage_params, int ctas) {
  std::ostringstream o;
  const int A = 1 << R;
  const int threads = 1 << (p.t - R);
  const int nw = std::max(1, threads / 32);
  const int ngrad = int(p.grad_slots.size());
  const TmaGeom& g = p.geom;
  const SharedMats smats = shared_mats(p, stage_params);
  o << kPrelude << shared_mats_decl(smats);
  o << "extern \"C\" __global__ void __launch_bounds__(" << threads << ", " << std::max(1, ctas)
    << ") mbk_adj(const __grid_constant__ TMap tmy, "
    << "const __grid_constant__ TMap tmd, const double2* __restrict__ tab, long long tstride, long long tps, "
    << "long long ntiles, u32* err, double* gpart, u32* gcount, double* gout, const int* __restrict__ gslot, "
    << "const double2* __restrict__ xtab) {\n";
  o << "  const double2* __restrict__ xtabs = nullptr; (void)xtabs;\n";
  o << "  extern __shared__ unsigned char smem_raw[];\n  __shared__ __align__(8) u64 bar[2];\n  __shared__ int s_abort;\n"
    << "  __shared__ bool lastcta;\n";
  o << shared_mats_fill(smats);
  const unsigned T = 1u << p.t;
  o << "  double2* base0 = (double2*)(((unsigned long long)smem_raw + 1023ull) & ~1023ull);\n";
  o << "  double2* ybuf[2] = {base0, base0 + " << T << "};\n  double2* dbuf[2] = {base0 + " << 2 * T << ", base0 + "
    << 3 * T << "};\n";
  o << "  double* gw = (double*)(base0 + " << 4 * T << ");\n";
  o << "  const u32 tx = threadIdx.x;\n";
  o << "  for (int i = tx; i < " << std::max(1, ngrad * nw) << "; i += blockDim.x) gw[i] = 0.0;\n";
  o << "  if (tx == 0) { mbar_init(&bar[0]); mbar_init(&bar[1]); asm volatile(\"fence.mbarrier_init.release.cluster;\" ::: \"memory\"); s_abort = 0; }\n";
  o << "  __syncthreads();\n";
  auto geom = [&](const char* tile, const char* pre) {
    std::ostringstream e;
    e << "  const int " << pre << "b = (int)(" << tile << " / tps);\n";
    e << "  u64 " << pre << "gb = (u64)(" << tile << " - (long long)" << pre << "b * tps);\n";
    for (int q = 0; q < p.t; ++q) {
      const int bit = p.bits[q];
      e << "  " << pre << "gb = ((" << pre << "gb >> " << bit << ") << " << (bit + 1) << ") | (" << pre << "gb & "
        << ((1ull << bit) - 1) << "ull);\n";
    }
    for (int d = 0; d < g.ndims; ++d) {
      e << "  const int " << pre << "c" << d << " = ";
      if (g.start[d] < 0) e << pre << "b;\n";
      else if (d == 0) e << "(int)(2ull * (" << pre << "gb & " << ((1ull << g.bits[0]) - 1) << "ull));\n";
      else e << "(int)((" << pre << "gb >> " << g.start[d] << ") & " << ((1ull << g.bits[d]) - 1) << "ull);\n";
    }
    return e.str();
  };
  auto subst = [&](std::string s, const char* pre, const char* map, const char* dst, const char* bar) {
    for (int d = 0; d < g.ndims && pre[0]; ++d) {
      const std::string from = "\"r\"(c" + std::to_string(d) + ")", to = std::string("\"r\"(") + pre + "c" + std::to_string(d) + ")";
      size_t pos;
      while ((pos = s.find(from)) != std::string::npos) s.replace(pos, from.size(), to);
    }
    size_t pos;
    while ((pos = s.find("&tmap")) != std::string::npos) s.replace(pos, 5, map);
    while ((pos = s.find("DST")) != std::string::npos) s.replace(pos, 3, dst);
    while ((pos = s.find("SRC")) != std::string::npos) s.replace(pos, 3, dst);
    while ((pos = s.find("BAR")) != std::string::npos) s.replace(pos, 3, bar);
    return s;
  };
  const std::string ld = tma_ld(g.ndims), st = tma_st(g.ndims);
  const unsigned bytes = 32u << p.t;  // y and delta tiles
  o << "  u32 ph0 = 0, ph1 = 0;\n  long long tile = blockIdx.x;\n";
  o << "  if (tx == 0 && tile < ntiles) {\n" << geom("tile", "p_") << "    mbar_tx(&bar[0], " << bytes << "u);\n    "
    << subst(ld, "p_", "&tmy", "ybuf[0]", "&bar[0]") << "\n    " << subst(ld, "p_", "&tmd", "dbuf[0]", "&bar[0]")
    << "\n  }\n";
  o << "  for (int it = 0; tile < ntiles; ++it, tile += gridDim.x) {\n    const int cur = it & 1;\n"
    << "    const long long nxt = tile + gridDim.x;\n";
  o << "    if (tx == 0 && nxt < ntiles) {\n" << geom("nxt", "n_")
    << "      asm volatile(\"cp.async.bulk.wait_group.read 0;\" ::: \"memory\");\n      mbar_tx(&bar[cur ^ 1], " << bytes
    << "u);\n      " << subst(ld, "n_", "&tmy", "ybuf[cur ^ 1]", "&bar[cur ^ 1]") << "\n      "
    << subst(ld, "n_", "&tmd", "dbuf[cur ^ 1]", "&bar[cur ^ 1]") << "\n    }\n";
  o << geom("tile", "");
  o << "    const double2* tb = tab + (long long)b * tstride;\n    (void)tb; (void)gb;\n";
  o << "    const double2* xb = xtabs; (void)xb;\n";
  o << "    double2* ty = ybuf[cur]; double2* td = dbuf[cur];\n";
  o << "    if (!mbar_wait(&bar[cur], cur ? ph1 : ph0)) { atomicOr(err, 1u); s_abort = 1; }\n";
  o << "    if (cur) ph1 ^= 1u; else ph0 ^= 1u;\n    __syncthreads();\n    if (s_abort) break;\n";
  o << "    double2 ";
  for (int j = 0; j < A; ++j) o << (j ? ", " : "") << "y" << j << ", d" << j;
  o << ";\n";
  for (size_t si = 0; si < p.stages.size(); ++si) {
    const StageDesc& sd = p.stages[si];
    o << "    {\n      const u32 lb = 0u";
    for (int q = 0; q < sd.ntid; ++q) o << " | (((tx >> " << q << ") & 1u) << " << sd.tid[q] << ")";
    o << ";\n";
    for (int j = 0; j < A; ++j)
      o << "      y" << j << " = ty[swz(lb | " << reg_off_const(j, R, sd.reg) << ")]; d" << j << " = td[swz(lb | "
        << reg_off_const(j, R, sd.reg) << ")];\n";
    StageGen gy{R, sd.reg, o, false, std::vector<int>(A), "y"};
    StageGen gd{R, sd.reg, o, false, std::vector<int>(A), "d"};
    gy.smap = gd.smap = &smats.slot;
    for (int j = 0; j < A; ++j) gy.nm[j] = gd.nm[j] = j;
    // gradient partial sums of this stage, reduced together in chunks (2 with 16 amplitudes per
    // thread, 8 with 8: few enough live sums to stay in registers)
    const int gchunk = R >= 4 ? 2 : 8;
    std::vector<std::string> gnames;
    int gacc0 = -1, gcount = 0;
    for (int q = 0; q < sd.nops; ++q) {
      const MOp& m = p.mops[sd.op0 + q];
      if (m.type == MOP_GRAD || m.type == MOP_GRADP) {
        if (int(gnames.size()) == gchunk || (gacc0 >= 0 && int(m.active) != gacc0 + int(gnames.size()))) {
          emit_grad_reduce(o, gnames, gacc0, nw);
          gnames.clear();
        }
        if (gnames.empty()) gacc0 = int(m.active);
        const std::string name = "gp" + std::to_string(gcount++);
        o << "      double " << name << ";\n";
        emit_grad(o, m, gy, gd, R, name);
        gnames.push_back(name);
      } else {
        if (m.only != 2) gy.emit(m);   // channels: S^-1 on y only, S' on delta only
        if (m.only != 1) gd.emit(m);
      }
    }
    if (!gnames.empty()) emit_grad_reduce(o, gnames, gacc0, nw);
    for (int j = 0; j < A; ++j)
      o << "      ty[swz(lb | " << reg_off_const(j, R, sd.reg) << ")] = " << gy.v(j) << "; td[swz(lb | "
        << reg_off_const(j, R, sd.reg) << ")] = " << gd.v(j) << ";\n";
    o << stage_sync(p, si) << "    }\n";
  }
  o << "    asm volatile(\"fence.proxy.async.shared::cta;\" ::: \"memory\");\n    __syncthreads();\n";
  o << "    if (tx == 0) { " << subst(st, "", "&tmy", "ty", "") << " " << subst(st, "", "&tmd", "td", "") << " }\n";
  o << "  }\n  if (tx == 0) asm volatile(\"cp.async.bulk.wait_group 0;\" ::: \"memory\");\n";
  // Gradient partials: per CTA, then the last CTA sums over CTAs in order.
  if (ngrad > 0) {
    o << "  __syncthreads();\n";
    o << "  for (int gi = tx; gi < " << ngrad << "; gi += blockDim.x) { double s = 0.0; for (int w = 0; w < " << nw
      << "; ++w) s += gw[gi * " << nw << " + w]; gpart[(long long)gi * gridDim.x + blockIdx.x] = s; }\n";
    o << "  __threadfence();\n  __syncthreads();\n";
    o << "  if (tx == 0) lastcta = atomicAdd(gcount, 1u) == gridDim.x - 1;\n  __syncthreads();\n";
    o << "  if (lastcta) {\n    __threadfence();\n    for (int gi = tx; gi < " << ngrad
      << "; gi += blockDim.x) { double s = 0.0; for (unsigned c = 0; c < gridDim.x; ++c) s += __ldcg(&gpart[(long long)gi * gridDim.x + c]); atomicAdd(&gout[gslot[gi]], s); }\n";
    o << "    __syncthreads();\n    if (tx == 0) *gcount = 0u;\n  }\n";
  }
  o << "}\n";
  (void)N;
  return o.str();
}

int jit_launch_adjoint(CUfunction fn, const CUtensorMap* my, const CUtensorMap* md, const double2* tab, int64_t tstride,
                       int64_t tps, int64_t ntiles, unsigned* err, double* gpart, unsigned* gcount, double* gout,
                       const int* gslot, const double2* xtab, int threads, size_t shm, int grid, cudaStream_t st) {
  Drv& d = drv();
  if (d.setattr(fn, CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES, int(shm)) != CUDA_SUCCESS) return MB_EDEVICE;
  long long ts = tstride, tp = tps, nt = ntiles;
  void* params[] = {(void*)my, (void*)md, (void*)&tab, &ts, &tp, &nt, &err, &gpart, &gcount, &gout, (void*)&gslot,
                    (void*)&xtab};
  if (d.launch(fn, grid, 1, 1, threads, 1, 1, unsigned(shm), (CUstream)st, params, nullptr) != CUDA_SUCCESS) {
    set_error("JIT adjoint launch failed");
    return MB_EDEVICE;
  }
  return MB_OK;
}

std::string jit_reg_source(const Pass& p, int N, bool stage_params) {
  std::ostringstream o;
  const int R = p.t, A = 1 << R;
  const SharedMats smats = shared_mats(p, stage_params);
  o << kPrelude << shared_mats_decl(smats);
  o << "extern \"C\" __global__ void __launch_bounds__(128) mbk_reg(double2* __restrict__ v, const double2* __restrict__ tab, "
    << "const double2* __restrict__ xtab, const double2* __restrict__ xtabs, long long xrow, long long tstride, "
    << "long long groups, int nsamples) {\n";
  if (!smats.offs.empty()) o << shared_mats_fill(smats) << "  __syncthreads();\n";
  o << "  const long long total = groups * nsamples;\n";
  o << "  for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < total; g += (long long)gridDim.x * blockDim.x) {\n";
  o << "    const int b = (int)(g / groups);\n    u64 lb = (u64)(g - (long long)b * groups);\n";
  for (int k = 0; k < R; ++k) {
    const int bit = p.bits[k];
    o << "    lb = ((lb >> " << bit << ") << " << (bit + 1) << ") | (lb & " << ((1ull << bit) - 1) << "ull);\n";
  }
  o << "    const u64 gb = 0ull; (void)gb;\n";
  o << "    double2* vs = v + ((long long)b << " << N << ");\n";
  o << "    const double2* tb = tab + (long long)b * tstride; (void)tb;\n";
  o << "    const double2* xb = xtabs + (long long)b * xrow; (void)xb;\n";
  int reg[kMaxRegBits];
  for (int k = 0; k < R; ++k) reg[k] = p.bits[k];
  for (int j = 0; j < A; ++j) o << "    double2 a" << j << " = vs[lb | " << reg_off_const(j, R, reg) << "];\n";
  StageGen sg{R, reg, o, true, std::vector<int>(A)};
  sg.smap = &smats.slot;
  for (int j = 0; j < A; ++j) sg.nm[j] = j;
  for (const MOp& m : p.mops) sg.emit(m);
  for (int j = 0; j < A; ++j) o << "    vs[lb | " << reg_off_const(j, R, reg) << "] = " << sg.v(j) << ";\n";
  o << "  }\n}\n";
  return o.str();
}

// ---- persistent uneven launch ----------------------------------------------------------------
// One kernel over samples of several register sizes: its work items are (pass, sample, chunk of
// tiles), ordered by pass index, taken from a work counter, each waiting on its sample's
// completion counter for the chunks of the previous pass (the protocol of the interpreter form
// k_uneven). Every pass is a straight-line device function of its own; the kernel dispatches an
// item to it with a switch. Functions are not inlined, so each is optimised and register-
// allocated on its own, and the module's compile time grows with the number of passes, not
// faster.

// Matrix elements of one pass for one sample, fixed and per-sample entries in one shared copy
// (per-sample keys carry kRowKey), filled once per work item. At most 2048 entries (32 KB); a
// pass with more reads its elements from the tables.
constexpr int32_t kRowKey = 1 << 28;
constexpr int32_t kKeyOff = kRowKey - 1;

static SharedMats uneven_mats(const Pass& p) {
  SharedMats sm;
  bool ok = true;
  auto add = [&](const MOp& m, int e) {
    if ((m.off[e] & ~kXtabFlag) > kKeyOff) ok = false;
    const int key = smat_key(m, e) | (m.param ? kRowKey : 0);
    if (sm.slot.count(key)) return;
    sm.slot[key] = int(sm.offs.size());
    sm.offs.push_back(key);
  };
  for (const MOp& m : p.mops) switch (m.type) {
      case MOP_U1: case MOP_CTRL: case MOP_RROT: case MOP_IROT: for (int e = 0; e < 4; ++e) add(m, e); break;
      case MOP_LIFT: add(m, 0); break;
      case MOP_U2: for (int e = 0; e < 16; ++e) add(m, e); break;
      case MOP_CHAN: for (int e = 0; e < 6; ++e) add(m, e); break;
      case MOP_DIAG: for (int e = 0; e < (1 << m.nsel); ++e) if ((m.active >> e) & 1) add(m, e); break;
      case MOP_CPHASE: if (!m.r1) add(m, 0); break;
      default: break;
    }
  if (!ok || sm.offs.size() > 2048) sm = SharedMats();
  return sm;
}

// Global offset of the pass-local index `l` (a u32 expression): every run of consecutive pass
// bits moves as one masked shift.
static std::string deposit_expr(const Pass& p, const char* l) {
  std::ostringstream e;
  e << "(0ull";
  for (int q = 0; q < p.t;) {
    int r = q + 1;
    while (r < p.t && p.bits[r] == p.bits[r - 1] + 1) ++r;
    e << " | ((u64)((" << l << " >> " << q << ") & " << ((1u << (r - q)) - 1) << "u) << " << p.bits[q] << ")";
    q = r;
  }
  e << ")";
  return e.str();
}

// Device function mbp<k>: every tile of one chunk of pass k for sample b (load through L2, the
// register stages, store).
static void emit_uneven_pass(std::ostringstream& o, const UnevenJitPass& up, int k, int R, int threads, int tmax) {
  const Pass& p = *up.p;
  const int A = 1 << R, T = 1 << p.t, vt = 1 << (p.t - R);
  const SharedMats sm = uneven_mats(p);
  if (!sm.offs.empty()) {
    o << "__constant__ int k_um" << k << "[" << sm.offs.size() << "] = {";
    for (size_t i = 0; i < sm.offs.size(); ++i) o << (i ? "," : "") << sm.offs[i];
    o << "};\n";
  }
  o << "static __device__ __noinline__ void mbp" << k << "(const UG* __restrict__ gd, int b, int chunk, int zero_init) {\n";
  o << "  const u32 tx = threadIdx.x;\n  double2* tl = dynsm;\n  double2* smat = dynsm + " << (1 << tmax)
    << "; (void)smat; (void)zero_init;\n";
  o << "  const UG G = *gd;\n  const double2* tab = G.table; const double2* xtab = G.xtab; (void)tab; (void)xtab;\n";
  o << "  const double2* tb = tab + (long long)b * G.tstride; const double2* xb = G.xtabs + (long long)b * G.xrow;"
    << " (void)tb; (void)xb;\n";
  o << "  double2* v = G.states + ((long long)b << " << up.n << ");\n";
  if (!sm.offs.empty())
    o << "  for (u32 i = tx; i < " << sm.offs.size() << "u; i += " << threads << "u) { const int mo = k_um" << k
      << "[i]; smat[i] = (mo & " << kXrowKey << ") ? __ldg(xb + (mo & " << kKeyOff << ")) : (mo & " << kRowKey
      << ") ? __ldg(tb + (mo & " << kKeyOff << ")) : (mo & " << kXtabFlag << ") ? __ldg(xtab + (mo & " << kKeyOff
      << ")) : __ldg(tab + mo); }\n";
  const long long ntiles = 1ll << (up.n - p.t);
  const long long per = (ntiles + up.nchunks - 1) / up.nchunks;
  o << "  const long long t0 = (long long)chunk * " << per << "ll;\n  const long long t1 = t0 + " << per << "ll < "
    << ntiles << "ll ? t0 + " << per << "ll : " << ntiles << "ll;\n";
  o << "  for (long long tile = t0; tile < t1; ++tile) {\n    u64 gb = (u64)tile;\n";
  std::vector<int> sorted(p.bits.begin(), p.bits.begin() + p.t);
  std::sort(sorted.begin(), sorted.end());
  for (int bit : sorted)
    o << "    gb = ((gb >> " << bit << ") << " << (bit + 1) << ") | (gb & " << ((1ull << bit) - 1) << "ull);\n";
  const std::string dep = deposit_expr(p, "l");
  o << "    for (u32 l = tx; l < " << T << "u; l += " << threads << "u) {\n      const u64 go = gb | " << dep << ";\n";
  if (up.first)
    o << "      tl[swz(l)] = zero_init ? make_double2(go == 0ull ? 1.0 : 0.0, 0.0) : __ldcg(v + go);\n";
  else
    o << "      tl[swz(l)] = __ldcg(v + go);\n";
  o << "    }\n    __syncthreads();\n    double2 ";
  for (int j = 0; j < A; ++j) o << (j ? ", " : "") << "a" << j;
  o << ";\n";
  for (size_t si = 0; si < p.stages.size(); ++si) {
    const StageDesc& sd = p.stages[si];
    o << "    " << (vt < threads ? "if (tx < " + std::to_string(vt) + "u) " : std::string()) << "{\n      const u32 lb = 0u";
    for (int q = 0; q < sd.ntid; ++q) o << " | (((tx >> " << q << ") & 1u) << " << sd.tid[q] << ")";
    o << ";\n";
    for (int j = 0; j < A; ++j) o << "      a" << j << " = tl[swz(lb | " << reg_off_const(j, R, sd.reg) << ")];\n";
    StageGen sg{R, sd.reg, o, false, std::vector<int>(A)};
    sg.smap = &sm.slot;
    sg.pkey = kRowKey;
    for (int j = 0; j < A; ++j) sg.nm[j] = j;
    for (int q = 0; q < sd.nops; ++q) sg.emit(p.mops[sd.op0 + q]);
    for (int j = 0; j < A; ++j) o << "      tl[swz(lb | " << reg_off_const(j, R, sd.reg) << ")] = " << sg.v(j) << ";\n";
    o << "    }\n" << stage_sync(p, si);
  }
  o << "    __syncthreads();\n    for (u32 l = tx; l < " << T << "u; l += " << threads << "u) v[gb | " << dep
    << "] = tl[swz(l)];\n    __syncthreads();\n  }\n}\n";
}

std::string jit_uneven_source(const std::vector<UnevenJitPass>& passes, int R, int ctas, int* threads, size_t* shm) {
  int tmax = R + 5;
  size_t ne = 0;
  for (const UnevenJitPass& up : passes) {
    tmax = std::max(tmax, up.p->t);
    ne = std::max(ne, uneven_mats(*up.p).offs.size());
  }
  const int th = 1 << (tmax - R);
  std::ostringstream o;
  o << kPrelude;
  o << "struct UG { double2* states; const double2* table; const double2* xtab; const double2* xtabs; "
    << "long long tstride; long long xrow; };\n";
  o << "extern __shared__ double2 dynsm[];\n";
  for (size_t k = 0; k < passes.size(); ++k) emit_uneven_pass(o, passes[k], int(k), R, th, tmax);
  o << "extern \"C\" __global__ void __launch_bounds__(" << th << ", " << std::max(1, ctas)
    << ") mbk_uneven(const UG* __restrict__ groups, const int4* __restrict__ pinfo, const int4* __restrict__ items, "
    << "int nitems, u32* next, u32* done, int zero_init, u32* err) {\n";
  o << "  __shared__ int s_item, s_ok;\n  const u32 tx = threadIdx.x;\n  for (;;) {\n";
  o << "    if (tx == 0) s_item = (int)atomicAdd(next, 1u);\n    __syncthreads();\n    const int item = s_item;\n"
    << "    if (item >= nitems) break;\n    const int4 it = items[item];\n    const int4 pi = pinfo[it.x];\n"
    << "    u32* cnt = done + pi.x + it.y;\n";
  // every chunk of the previous passes of this sample (taken earlier by running CTAs)
  o << "    if (tx == 0) {\n      int ok = 1;\n"
    << "      for (u32 spin = 0; atomicAdd(cnt, 0u) < (u32)pi.y; ++spin) {\n"
    << "        if (spin > (1u << 24)) { atomicOr(err, 1u); ok = 0; break; }\n        __nanosleep(64);\n      }\n"
    << "      __threadfence();\n      s_ok = ok;\n    }\n    __syncthreads();\n    if (!s_ok) break;\n";
  o << "    switch (it.x) {\n";
  for (size_t k = 0; k < passes.size(); ++k)
    o << "      case " << k << ": mbp" << k << "(groups + pi.z, it.y, it.z, zero_init); break;\n";
  o << "      default: break;\n    }\n";
  // publish this chunk: every thread's stores, then the counter
  o << "    __threadfence();\n    __syncthreads();\n    if (tx == 0) atomicAdd(cnt, 1u);\n  }\n}\n";
  *threads = th;
  *shm = (size_t(16) << tmax) + 16 * ne;
  return o.str();
}

int jit_launch_uneven(CUfunction fn, const UnevenJitGroup* groups, const int4* pinfo, const int4* items, int nitems,
                      unsigned* next, unsigned* done, int zero_init, unsigned* err, int threads, size_t shm, int grid,
                      cudaStream_t st) {
  Drv& d = drv();
  if (d.setattr(fn, CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES, int(shm)) != CUDA_SUCCESS) return MB_EDEVICE;
  int ni = nitems, zi = zero_init;
  void* params[] = {(void*)&groups, (void*)&pinfo, (void*)&items, &ni, &next, &done, &zi, &err};
  if (d.launch(fn, grid, 1, 1, threads, 1, 1, unsigned(shm), (CUstream)st, params, nullptr) != CUDA_SUCCESS) {
    set_error("persistent uneven launch failed");
    return MB_EDEVICE;
  }
  return MB_OK;
}

// ---- Pauli-string expectation pass -------------------------------------------------------------
// The pass of k_pauli_pass (tiles of the five lane bits and nr register bits in shared memory,
// every flip group of the pass evaluated against its partner amplitudes) with the groups,
// their flip masks and the strings' Z masks as constants. A string's sign at index
// j = base | l splits into a tile-base part (-1)^{|base & zh|} and a local part
// (-1)^{|(l ^ x) & zl|}; strings of a group with the same zh form a class whose local sum
// F(l) = sum_s c_s (-1)^{|(l ^ x) & zl_s|} depends only on the thread's own local indices, so it
// is formed once per thread before the tile loop and each tile costs one sign per class.
// Coefficients come from an array, so observables that differ only in them share the kernel.

// Global bits of local index `e` (a u32 expression): lane bits 0..4, then register bits.
static std::string pauli_local_bits(const PauliJitPass& p, const std::string& e) {
  std::ostringstream o;
  o << "((u64)((" << e << ") & 31u)";
  for (int r = 0; r < p.nr;) {
    int q = r + 1;
    while (q < p.nr && p.reg[q] == p.reg[q - 1] + 1) ++q;
    o << " | ((u64)(((" << e << ") >> " << (5 + r) << ") & " << ((1u << (q - r)) - 1) << "u) << " << p.reg[r] << ")";
    r = q;
  }
  o << ")";
  return o.str();
}

std::string jit_pauli_source(const PauliJitPass& p, int max_vals) {
  constexpr int kThreads = 256;
  const int local = 5 + p.nr, per = (1 << local) / kThreads;
  uint64_t localm = 31;
  for (int r = 0; r < p.nr; ++r) localm |= uint64_t(1) << p.reg[r];
  // classes of every group (strings with the same zh); a class is real when all of its
  // coefficients are, and local when some string has Z bits among the local bits
  struct Cls {
    uint64_t zh;
    std::vector<PauliJitString> s;
    bool local, real;
  };
  std::vector<std::vector<Cls>> cls(p.groups.size());
  std::vector<bool> greal(p.groups.size(), true);
  int vals = 0;
  for (size_t g = 0; g < p.groups.size(); ++g) {
    const PauliJitGroup& G = p.groups[g];
    std::map<uint64_t, size_t> at;
    for (const PauliJitString& s : G.strings) {
      const uint64_t zh = s.z & ~localm;
      if (!at.count(zh)) {
        at[zh] = cls[g].size();
        cls[g].push_back(Cls{zh, {}, false, true});
      }
      Cls& c = cls[g][at[zh]];
      c.s.push_back(s);
      c.local = c.local || (s.z & localm) != 0;
      c.real = c.real && s.real;
    }
    const int slots = (G.xl != 0 && G.herm) ? per / 2 : per;
    for (const Cls& c : cls[g]) {
      if (c.local) vals += slots * (c.real ? 1 : 2);
      greal[g] = greal[g] && c.real;
    }
  }
  if (vals > max_vals) return "";
  auto fname = [](size_t g, size_t c, int k) {
    return "F" + std::to_string(g) + "_" + std::to_string(c) + "_" + std::to_string(k);
  };
  std::ostringstream o;
  o << kPrelude;
  o << "__device__ __forceinline__ double dneg(double a, u64 s) { return __longlong_as_double(__double_as_longlong(a) ^ "
       "(long long)s); }\n";
  o << "extern \"C\" __global__ void __launch_bounds__(" << kThreads << ", " << std::max(1, std::min(4, p.ctas))
    << ") mbk_pauli(const double2* __restrict__ v, "
    << "const double2* __restrict__ coef, long long tps, double2* partials, u32* counters, double2* out) {\n";
  o << "  extern __shared__ double2 tile[];\n  __shared__ double2 wp[" << kThreads / 32 << "];\n  __shared__ bool last;\n";
  o << "  const u32 tx = threadIdx.x;\n  const int b = blockIdx.y, G = gridDim.x;\n";
  o << "  const double2* vs = v + ((long long)b << " << p.n << ");\n";
  for (int k = 0; k < per; ++k)
    o << "  const u64 lk" << k << " = " << pauli_local_bits(p, "tx + " + std::to_string(k * kThreads) + "u") << ";\n";
  auto idx = [&](size_t g, int k) {
    const PauliJitGroup& G = p.groups[g];
    return (G.xl != 0 && G.herm) ? "i" + std::to_string(g) + "_" + std::to_string(k)
                                 : "(tx + " + std::to_string(k * kThreads) + "u)";
  };
  auto lbits = [&](size_t g, int k) {
    const PauliJitGroup& G = p.groups[g];
    return (G.xl != 0 && G.herm) ? "b" + std::to_string(g) + "_" + std::to_string(k) : "lk" + std::to_string(k);
  };
  // factors of the local classes at the thread's own local indices (Hermitian flip groups: the
  // pair members with bit hb clear)
  for (size_t g = 0; g < p.groups.size(); ++g) {
    const PauliJitGroup& G = p.groups[g];
    const bool herm = G.xl != 0 && G.herm;
    const int slots = herm ? per / 2 : per;
    if (herm)
      for (int k = 0; k < slots; ++k) {
        const std::string m = "(tx + " + std::to_string(k * kThreads) + "u)";
        const std::string nm = "i" + std::to_string(g) + "_" + std::to_string(k);
        o << "  const u32 " << nm << " = ((" << m << " >> " << G.hb << ") << " << (G.hb + 1) << ") | (" << m << " & "
          << ((1u << G.hb) - 1) << "u);\n";
        o << "  const u64 b" << g << "_" << k << " = " << pauli_local_bits(p, nm) << ";\n";
      }
    for (size_t c = 0; c < cls[g].size(); ++c) {
      const Cls& C = cls[g][c];
      if (!C.local) continue;
      for (int k = 0; k < slots; ++k) {
        const std::string F = fname(g, c, k);
        o << "  " << (C.real ? "double " : "double2 ") << F << (C.real ? " = 0.0;\n" : " = make_double2(0.0, 0.0);\n");
        for (const PauliJitString& s : C.s) {
          const uint64_t zl = s.z & localm;
          const std::string q = "__ldg(coef + " + std::to_string(s.s) + ")";
          const std::string sg = "(u64)(__popcll((" + lbits(g, k) + " ^ " + std::to_string(G.x) + "ull) & " +
                                 std::to_string(zl) + "ull) & 1) << 63";
          if (C.real)
            o << "  " << F << " += " << (zl ? "dneg(" + q + ".x, " + sg + ")" : q + ".x") << ";\n";
          else
            o << "  { const double2 t = " << (zl ? "cneg(" + q + ", " + sg + ")" : q) << "; " << F << ".x += t.x; " << F
              << ".y += t.y; }\n";
        }
      }
    }
  }
  // Tiles of 2^10 amplitudes are double-buffered: each thread's asynchronous copies of the next
  // tile (cp.async, 16 bytes each) are in flight while the block evaluates the current one.
  const bool dbl = pauli_jit_shm(p.nr) > (size_t(16) << local);
  std::vector<int> regs(p.reg, p.reg + p.nr);
  std::sort(regs.begin(), regs.end());
  auto tbase = [&](const std::string& t, const std::string& name) {
    std::ostringstream e;
    e << "    u64 " << name << " = (u64)(" << t << ") << 5;\n";
    for (int bit : regs)
      e << "    " << name << " = ((" << name << " >> " << bit << ") << " << (bit + 1) << ") | (" << name << " & "
        << ((1ull << bit) - 1) << "ull);\n";
    return e.str();
  };
  auto fetch = [&](const std::string& buf, const std::string& bname) {
    std::ostringstream e;
    for (int k = 0; k < per; ++k)
      e << "      asm volatile(\"cp.async.cg.shared.global [%0], [%1], 16;\" :: \"r\"(sa(" << buf << " + tx + "
        << k * kThreads << "u)), \"l\"(vs + (" << bname << " | lk" << k << ")) : \"memory\");\n";
    return e.str();
  };
  o << "  double ar = 0.0, ai = 0.0;\n";
  if (dbl) {
    o << "  int it = 0;\n  if ((long long)blockIdx.x < tps) {\n" << tbase("blockIdx.x", "nb") << fetch("tile", "nb")
      << "  }\n  asm volatile(\"cp.async.commit_group;\" ::: \"memory\");\n";
    o << "  for (long long T = blockIdx.x; T < tps; T += G, ++it) {\n";
    o << "    double2* const cur = tile + (it & 1) * " << (1 << local) << ";\n";
    o << "    if (T + G < tps) {\n" << tbase("T + G", "nb") << fetch("tile + ((it + 1) & 1) * " + std::to_string(1 << local), "nb")
      << "    }\n";
    o << "    asm volatile(\"cp.async.commit_group;\" ::: \"memory\");\n"
      << "    asm volatile(\"cp.async.wait_group 1;\" ::: \"memory\");\n";
    o << tbase("T", "base");
  } else {
    o << "  for (long long T = blockIdx.x; T < tps; T += G) {\n    double2* const cur = tile;\n" << tbase("T", "base");
    for (int k = 0; k < per; ++k) o << "    tile[tx + " << k * kThreads << "u] = vs[base | lk" << k << "];\n";
  }
  o << "    __syncthreads();\n";
  for (size_t g = 0; g < p.groups.size(); ++g) {
    const PauliJitGroup& G = p.groups[g];
    const bool herm = G.xl != 0 && G.herm, re = greal[g];
    const int slots = herm ? per / 2 : per;
    // classes without local Z bits: one value per tile (coefficients read through the cache)
    o << "    {\n      double kx = 0.0" << (re ? "" : ", ky = 0.0") << ";\n";
    for (size_t c = 0; c < cls[g].size(); ++c) {
      const Cls& C = cls[g][c];
      const std::string sg = "(u64)(__popcll(base & " + std::to_string(C.zh) + "ull) & 1) << 63";
      if (C.local) {
        if (C.zh) o << "      const u64 s" << c << " = " << sg << ";\n";
        continue;
      }
      o << "      { double2 t = make_double2(0.0, 0.0);";
      for (const PauliJitString& s : C.s) o << " { const double2 q = __ldg(coef + " << s.s << "); t.x += q.x; t.y += q.y; }";
      if (C.zh) o << " t = cneg(t, " << sg << ");";
      o << " kx += t.x;" << (re ? "" : " ky += t.y;") << " }\n";
    }
    for (int k = 0; k < slots; ++k) {
      o << "      { double fx = kx" << (re ? "" : ", fy = ky") << ";\n";
      for (size_t c = 0; c < cls[g].size(); ++c) {
        const Cls& C = cls[g][c];
        if (!C.local) continue;
        const std::string F = fname(g, c, k), s = "s" + std::to_string(c);
        if (C.real)
          o << "        fx += " << (C.zh ? "dneg(" + F + ", " + s + ")" : F) << ";\n";
        else
          o << "        { const double2 t = " << (C.zh ? "cneg(" + F + ", " + s + ")" : F) << "; fx += t.x; fy += t.y; }\n";
      }
      const std::string i = idx(g, k), av = "cur[" + i + "]";
      if (G.xl == 0) {
        o << "        const double2 a = " << av << "; const double p2 = fma(a.x, a.x, a.y * a.y);\n"
          << "        ar = fma(fx, p2, ar);" << (re ? "" : " ai = fma(fy, p2, ai);") << " }\n";
      } else {
        o << "        const double2 a = " << av << ", q = cur[" << i << " ^ " << G.xl << "u];\n"
          << "        const double cr = fma(a.x, q.x, a.y * q.y), ci = fma(a.x, q.y, -a.y * q.x); (void)ci;\n";
        if (herm)
          o << "        ar = fma(2.0 * fx, cr, " << (re ? "ar" : "fma(-2.0 * fy, ci, ar)") << "); }\n";
        else if (re)
          o << "        ar = fma(fx, cr, ar); ai = fma(fx, ci, ai); }\n";
        else
          o << "        ar = fma(fx, cr, fma(-fy, ci, ar)); ai = fma(fx, ci, fma(fy, cr, ai)); }\n";
      }
    }
    o << "    }\n";
  }
  o << "    __syncthreads();\n  }\n";
  if (dbl) o << "  asm volatile(\"cp.async.wait_all;\" ::: \"memory\");\n";
  // block sum, then the last block of the sample adds the blocks' sums in block order
  o << "  for (int d = 16; d > 0; d >>= 1) { ar += __shfl_down_sync(0xffffffffu, ar, d); "
    << "ai += __shfl_down_sync(0xffffffffu, ai, d); }\n";
  o << "  if ((tx & 31u) == 0u) wp[tx >> 5] = make_double2(ar, ai);\n  __syncthreads();\n";
  o << "  if (tx == 0) {\n    double sx = 0.0, sy = 0.0;\n    for (int w = 0; w < " << kThreads / 32
    << "; ++w) { sx += wp[w].x; sy += wp[w].y; }\n"
    << "    partials[(long long)b * G + blockIdx.x] = make_double2(sx, sy);\n    __threadfence();\n"
    << "    last = atomicAdd(&counters[b], 1u) == (u32)(G - 1);\n  }\n  __syncthreads();\n";
  o << "  if (last && tx == 0) {\n    double sx = 0.0, sy = 0.0;\n"
    << "    for (int g = 0; g < G; ++g) { const double2 q = __ldcg(&partials[(long long)b * G + g]); sx += q.x; sy += q.y; }\n"
    << "    const double2 o0 = __ldcg(&out[b]);\n    out[b] = make_double2(o0.x + sx, o0.y + sy);\n"
    << "    counters[b] = 0;\n  }\n}\n";
  return o.str();
}

int jit_launch_pauli(CUfunction fn, const double2* v, const double2* coef, int64_t tps, double2* partials,
                     unsigned* counters, double2* out, int grid, int batch, size_t shm, cudaStream_t st) {
  Drv& d = drv();
  if (d.setattr(fn, CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES, int(shm)) != CUDA_SUCCESS) return MB_EDEVICE;
  long long tp = tps;
  void* params[] = {(void*)&v, (void*)&coef, &tp, &partials, &counters, &out};
  if (d.launch(fn, grid, batch, 1, 256, 1, 1, unsigned(shm), (CUstream)st, params, nullptr) != CUDA_SUCCESS) {
    set_error("specialised Pauli pass launch failed");
    return MB_EDEVICE;
  }
  return MB_OK;
}

int jit_prepare(std::vector<std::string>& sources, std::vector<CUfunction>& out, std::string* err, double budget_s) {
  out.assign(sources.size(), nullptr);
  // kernels already compiled are taken here; worker threads start only for the others
  std::vector<size_t> todo;
  {
    std::lock_guard<std::mutex> lk(g_jit_mu);
    for (size_t i = 0; i < sources.size(); ++i) {
      auto it = g_cache.find(sources[i]);
      if (it != g_cache.end()) {
        out[i] = it->second.fn;
        it->second.last = ++g_tick;
      } else {
        todo.push_back(i);
      }
    }
  }
  if (todo.empty()) return MB_OK;
  std::vector<std::string> errs(sources.size());
  std::vector<char> skipped(sources.size(), 0);
  std::vector<std::thread> pool;
  const size_t nthreads = std::max<size_t>(1, std::min<size_t>(todo.size(), std::thread::hardware_concurrency()));
  // Compilation runs on worker threads; modules load on the worker threads too, which is
  // fine because the runtime's primary context is current on every thread of the process.
  int dev = 0;
  cudaGetDevice(&dev);
  std::atomic<size_t> next{0};
  const auto t0 = std::chrono::steady_clock::now();
  auto elapsed = [&] { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); };
  for (size_t w = 0; w < nthreads; ++w)
    pool.emplace_back([&] {
      cudaSetDevice(dev);
      cudaFree(nullptr);
      for (size_t j = next++; j < todo.size(); j = next++) {
        const size_t i = todo[j];
        // Past the budget only kernels already in the cache are taken; the rest run interpreted.
        if (budget_s > 0 && elapsed() > budget_s) {
          std::lock_guard<std::mutex> lk(g_jit_mu);
          auto it = g_cache.find(sources[i]);
          if (it != g_cache.end()) {
            out[i] = it->second.fn;
            it->second.last = ++g_tick;
          } else {
            skipped[i] = 1;
          }
          continue;
        }
        out[i] = compile_kernel(sources[i], &errs[i]);
      }
    });
  for (auto& t : pool) t.join();
  for (size_t i = 0; i < sources.size(); ++i)
    if (!out[i] && !skipped[i]) {
      *err = errs[i];
      return MB_EUNSUPPORTED;
    }
  return MB_OK;
}

int jit_launch_tile(CUfunction fn, const CUtensorMap* map, const double2* tab, const double2* xtab, const double2* xtabs,
                    int64_t xrow, int64_t tstride, int64_t tps, int64_t ntiles, unsigned* err, int threads, size_t shm,
                    int grid, cudaStream_t st) {
  Drv& d = drv();
  if (d.setattr(fn, CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES, int(shm)) != CUDA_SUCCESS) return MB_EDEVICE;
  long long ts = tstride, tp = tps, nt = ntiles;
  long long xr = xrow;
  void* params[] = {(void*)map, (void*)&tab, (void*)&xtab, (void*)&xtabs, &xr, &ts, &tp, &nt, &err};
  if (d.launch(fn, grid, 1, 1, threads, 1, 1, unsigned(shm), (CUstream)st, params, nullptr) != CUDA_SUCCESS) {
    set_error("JIT tile launch failed");
    return MB_EDEVICE;
  }
  return MB_OK;
}

int jit_launch_reg(CUfunction fn, double2* v, const double2* tab, const double2* xtab, const double2* xtabs,
                   int64_t xrow, int64_t tstride, int64_t groups, int nsamples, int grid, cudaStream_t st) {
  Drv& d = drv();
  long long ts = tstride, gr = groups;
  int ns = nsamples;
  long long xr = xrow;
  void* params[] = {&v, (void*)&tab, (void*)&xtab, (void*)&xtabs, &xr, &ts, &gr, &ns};
  if (d.launch(fn, grid, 1, 1, 128, 1, 1, 0, (CUstream)st, params, nullptr) != CUDA_SUCCESS) {
    set_error("JIT sweep launch failed");
    return MB_EDEVICE;
  }
  return MB_OK;
}

}  // namespace mb
