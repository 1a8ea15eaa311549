// NVRTC-specialised pass kernels (jit.cu).
#pragma once
#include <cuda.h>

#include <string>
#include <vector>

#include "fused.h"

namespace mb {
bool jit_available();
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
int jit_launch_reg(CUfunction fn, double2* v, const double2* tab, const double2* xtab, const double2* xtabs,
                   int64_t xrow, int64_t tstride, int64_t groups, int nsamples, int grid, cudaStream_t st);
}  // namespace mb
