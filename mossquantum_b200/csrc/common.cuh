// Shared internals of libmossb200 (host + device). Not part of the public ABI.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <string>

#include "../../include/mossb200.h"

namespace mb {

// ---------------------------------------------------------------------------------------
// Complex helpers on double2 (x = re, y = im), the device image of ComplexF64.
// ---------------------------------------------------------------------------------------
__host__ __device__ __forceinline__ double2 cz() { return make_double2(0.0, 0.0); }
__host__ __device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a*b + c with fused multiply-adds (4 FP64 instructions).
__host__ __device__ __forceinline__ double2 cfma(double2 a, double2 b, double2 c) {
  return make_double2(fma(a.x, b.x, fma(-a.y, b.y, c.x)), fma(a.x, b.y, fma(a.y, b.x, c.y)));
}
// conj(a)*b + c
__host__ __device__ __forceinline__ double2 cfma_conj(double2 a, double2 b, double2 c) {
  return make_double2(fma(a.x, b.x, fma(a.y, b.y, c.x)), fma(a.x, b.y, fma(-a.y, b.x, c.y)));
}
__host__ __device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
__host__ __device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }

// Matrix access modes: how a kernel reads the stored ordered matrix m (column-major, d x d).
enum MatMode : int {
  MAT_PLAIN = 0,      // m[r, c]
  MAT_CONJ = 1,       // conj(m[r, c])          (U on density-matrix column bits)
  MAT_ADJOINT = 2,    // conj(m[c, r])          (U')
  MAT_TRANSPOSE = 3,  // m[c, r]                (conj(U') on column bits)
};

__host__ __device__ __forceinline__ double2 mat_at(const double2* m, int d, int r, int c, int mode) {
  switch (mode) {
    case MAT_CONJ: return cconj(m[r + c * d]);
    case MAT_ADJOINT: return cconj(m[c + r * d]);
    case MAT_TRANSPOSE: return m[c + r * d];
    default: return m[r + c * d];
  }
}

// Insert a zero bit at each ascending position pos[0..k-1] into compact index i.
__host__ __device__ __forceinline__ int64_t insert_zeros(int64_t i, int k, const int* pos) {
  for (int j = 0; j < k; ++j) {
    int64_t low = i & ((int64_t(1) << pos[j]) - 1);
    i = ((i >> pos[j]) << (pos[j] + 1)) | low;
  }
  return i;
}

// Positions of a local operator, passed by value to kernels.
struct Pos {
  int k;
  int p[10];
};

// ---------------------------------------------------------------------------------------
// Host-side error handling and launch accounting
// ---------------------------------------------------------------------------------------
void set_error(const char* fmt, ...);
uint64_t& launch_counter();

#define MB_CHECK_CUDA(expr)                                                        \
  do {                                                                             \
    cudaError_t _e = (expr);                                                       \
    if (_e != cudaSuccess) {                                                       \
      ::mb::set_error("CUDA error %s at %s:%d: %s", cudaGetErrorName(_e), __FILE__, \
                      __LINE__, cudaGetErrorString(_e));                           \
      return MB_EDEVICE;                                                           \
    }                                                                              \
  } while (0)

#define MB_LAUNCHED()                                                  \
  do {                                                                 \
    ++::mb::launch_counter();                                          \
    cudaError_t _e = cudaGetLastError();                               \
    if (_e != cudaSuccess) {                                           \
      ::mb::set_error("kernel launch failed at %s:%d: %s", __FILE__,  \
                      __LINE__, cudaGetErrorString(_e));               \
      return MB_EDEVICE;                                               \
    }                                                                  \
  } while (0)

// Records a kernel launch in the optional per-kernel profile (CUDA events on `st`).
// Construct immediately before the launch and let it go out of scope right after.
struct ProfScope {
  int slot;
  cudaStream_t st;
  ProfScope(const char* name, double bytes, cudaStream_t stream, double flops = 0);
  ~ProfScope();
};

inline int grid_for(int64_t work, int block, int64_t cap = int64_t(148) * 32) {
  int64_t g = (work + block - 1) / block;
  if (g < 1) g = 1;
  if (g > cap) g = cap;
  return int(g);
}

}  // namespace mb
