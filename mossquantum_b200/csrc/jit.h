// NVRTC-specialised pass kernels (jit.cu).
#pragma once
#include <cuda.h>

#include <string>
#include <vector>

#include "fused.h"

namespace mb {
bool jit_available();
// Local memory (register spills, stack) per thread of a compiled kernel, or -1 if unknown.
int jit_local_bytes(void* fn);
// Reference counts of the compiled kernels a schedule uses; jit_trim unloads unreferenced
// modules beyond the cache cap (MB_JIT_CACHE_MAX).
void jit_retain(void* fn);
void jit_release(void* fn);
void jit_trim();
// Cumulative compile time (NVRTC and module load), compilations, modules loaded.
void jit_stats(double* compile_ms, uint64_t* compiles, size_t* modules);
// ctas: CTAs per SM the kernel is compiled for (its launch bounds; the launch uses the same).
std::string jit_tile_source(const Pass& p, int R, int N, bool stage_params, int ctas = 1);
std::string jit_reg_source(const Pass& p, int N, bool stage_params);
// Compiles every source (in parallel, cached by text); fills out[i] or fails with err. With a
// positive budget (seconds) sources not started within it are skipped (out[i] = nullptr) and
// the call still succeeds; a source that fails to compile always fails the call.
int jit_prepare(std::vector<std::string>& sources, std::vector<CUfunction>& out, std::string* err,
                double budget_s = 0);
int jit_launch_tile(CUfunction fn, const CUtensorMap* map, const double2* tab, const double2* xtab, const double2* xtabs,
                    int64_t xrow, int64_t tstride, int64_t tps, int64_t ntiles, unsigned* err, int threads, size_t shm,
                    int grid, cudaStream_t st);
std::string jit_adjoint_source(const Pass& p, int R, int N, bool stage_params, int ctas = 1);
int jit_launch_adjoint(CUfunction fn, const CUtensorMap* my, const CUtensorMap* md, const double2* tab, int64_t tstride,
                       int64_t tps, int64_t ntiles, unsigned* err, double* gpart, unsigned* gcount, double* gout,
                       const int* gslot, const double2* xtab, int threads, size_t shm, int grid, cudaStream_t st);
// One pass of a persistent uneven launch (mbk_uneven).
struct UnevenJitPass {
  const Pass* p;
  int n;          // amplitude bits of one sample
  bool first;     // pass 0 of its size: generates |0..0> when the launch asks for it
  int nchunks;    // work items per pass and sample
};
// Per-size descriptor mbk_uneven reads (the generated source declares the same layout).
struct UnevenJitGroup {
  double2* states;        // samples back to back
  const double2* table;   // matrix table, one row of tstride entries per sample
  const double2* xtab;    // derived coefficients
  const double2* xtabs;   // per-sample rows of xrow derived entries
  long long tstride, xrow;
};
static_assert(sizeof(UnevenJitGroup) == 48, "UnevenJitGroup layout is mirrored in generated code");
// Source of the persistent kernel over `passes` (item x of a launch names passes[x]) with
// register width R, compiled for `ctas` CTAs per SM; returns its threads per CTA and dynamic
// shared memory.
std::string jit_uneven_source(const std::vector<UnevenJitPass>& passes, int R, int ctas, int* threads, size_t* shm);
// pinfo[x] = (first completion counter of pass x's samples, chunks before pass x, group, 0);
// items[i] = (pass, sample, chunk, 0).
int jit_launch_uneven(CUfunction fn, const UnevenJitGroup* groups, const int4* pinfo, const int4* items, int nitems,
                      unsigned* next, unsigned* done, int zero_init, unsigned* err, int threads, size_t shm, int grid,
                      cudaStream_t st);
// One pass of a Pauli-string expectation (pauli.cu) for a specialised kernel (mbk_pauli): the
// pass's register bits and its flip groups with their strings (coefficient index, Z mask).
struct PauliJitString {
  int s;
  uint64_t z;
  bool real;   // the coefficient (with i^{#Y}) has no imaginary part
};
struct PauliJitGroup {
  uint64_t x;
  int xl, herm, hb;
  std::vector<PauliJitString> strings;
};
struct PauliJitPass {
  int n, nr;
  int reg[7];
  std::vector<PauliJitGroup> groups;
  int ctas = 3;   // CTAs per SM the kernel's registers are bounded for
};
// Source of the pass, or "" when its per-thread factors need more than max_vals registers of
// doubles (the interpreter kernel then runs the pass).
std::string jit_pauli_source(const PauliJitPass& p, int max_vals);
// Dynamic shared memory of a specialised Pauli pass: two tiles (double-buffered) of 2^(5+nr)
// amplitudes up to nr = 5, one above.
inline size_t pauli_jit_shm(int nr) { return (size_t(16) << (5 + nr)) * (nr <= 5 ? 2 : 1); }
int jit_launch_pauli(CUfunction fn, const double2* v, const double2* coef, int64_t tps, double2* partials,
                     unsigned* counters, double2* out, int grid, int batch, size_t shm, cudaStream_t st);
int jit_launch_reg(CUfunction fn, double2* v, const double2* tab, const double2* xtab, const double2* xtabs,
                   int64_t xrow, int64_t tstride, int64_t groups, int nsamples, int grid, cudaStream_t st);
}  // namespace mb
