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
      auto it = smap->find(smat_key(m, e));
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

// Entry point of a generated source: mbk_tile (tile pass), mbk_reg (strided sweep) or
// mbk_adj (adjoint dual-state pass).
const char* kernel_name(const std::string& src) {
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

int jit_prepare(std::vector<std::string>& sources, std::vector<CUfunction>& out, std::string* err, double budget_s) {
  out.assign(sources.size(), nullptr);
  std::vector<std::string> errs(sources.size());
  std::vector<char> skipped(sources.size(), 0);
  std::vector<std::thread> pool;
  const size_t nthreads = std::max<size_t>(1, std::min<size_t>(sources.size(), std::thread::hardware_concurrency()));
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
      for (size_t i = next++; i < sources.size(); i = next++) {
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
