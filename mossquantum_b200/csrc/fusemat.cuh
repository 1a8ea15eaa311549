// Bind-time fusion of consecutive operations on one qubit (host and device).
//
// A run of operations that act only on qubit q (pure states: bit q; density matrices: the row
// bit q and the column bit q + n) multiplies into one 2x2 (pure) or 4x4 (density) matrix. For
// fixed operations the product is formed once on the host; when a member is parametric it is
// formed per sample, right after parameter binding, by k_fuse (fused.cu). The passes then apply
// one dense micro-op instead of the run.
#pragma once
#include <cstdint>

#include "common.cuh"

namespace mb {

enum FuseKind : int8_t {
  FC_DENSE2 = 0,  // 2x2 from off[0..3] (column-major), on local bit `bit`
  FC_DIAG2 = 1,   // diag(off[0], off[1]) on local bit `bit`; entries outside `active` are 1
  FC_PHASE2 = 2,  // diag(1, off[0]) on local bit `bit` (diag(1, -1) when neg)
  FC_DENSE4 = 3,  // 4x4 from off[0..15] on local bits (0, 1)
};

struct FuseComp {
  int8_t kind;
  int8_t bit;     // local bit of a 2x2 component inside a 4x4 product
  int8_t conj;    // read the entries conjugated
  int8_t param;   // entries of the sample's own table row (else row 0)
  int8_t neg;     // FC_PHASE2: factor -1
  uint8_t active; // FC_DIAG2
  int16_t pad;
  int32_t off[16];
};

struct FuseRec {
  int32_t out;    // first entry of the product in a sample's row of the derived table
  int32_t d;      // 2 or 4
  int32_t c0, nc; // components [c0, c0 + nc) in application order
};

// M (d x d, column-major) = product of the record's components, the last one leftmost.
__host__ __device__ inline void fuse_product(const FuseRec& r, const FuseComp* comps, const double2* row0,
                                             const double2* rowb, double2* M) {
  const int d = r.d;
  for (int i = 0; i < d * d; ++i) M[i] = make_double2((i % (d + 1)) == 0 ? 1.0 : 0.0, 0.0);
  for (int ci = 0; ci < r.nc; ++ci) {
    const FuseComp& c = comps[r.c0 + ci];
    const double2* src = c.param ? rowb : row0;
    auto el = [&](int e) {
      const double2 v = src[c.off[e]];
      return c.conj ? make_double2(v.x, -v.y) : v;
    };
    if (c.kind == FC_DENSE4) {
      double2 X[16], T[16];
      for (int e = 0; e < 16; ++e) X[e] = el(e);
      for (int row = 0; row < 4; ++row)
        for (int col = 0; col < 4; ++col) {
          double2 acc = cz();
          for (int k = 0; k < 4; ++k) acc = cfma(X[row + 4 * k], M[k + 4 * col], acc);
          T[row + 4 * col] = acc;
        }
      for (int e = 0; e < 16; ++e) M[e] = T[e];
      continue;
    }
    double2 x00, x10, x01, x11;
    if (c.kind == FC_DENSE2) {
      x00 = el(0);
      x10 = el(1);
      x01 = el(2);
      x11 = el(3);
    } else if (c.kind == FC_DIAG2) {
      x00 = (c.active & 1) ? el(0) : make_double2(1.0, 0.0);
      x11 = (c.active & 2) ? el(1) : make_double2(1.0, 0.0);
      x10 = x01 = cz();
    } else {
      x00 = make_double2(1.0, 0.0);
      x11 = c.neg ? make_double2(-1.0, 0.0) : el(0);
      x10 = x01 = cz();
    }
    // rows of M along local bit `bit`: [M[r0, col], M[r1, col]] <- X [M[r0, col], M[r1, col]]
    const int b = d == 2 ? 1 : (1 << c.bit);
    for (int col = 0; col < d; ++col)
      for (int r0 = 0; r0 < d; ++r0) {
        if (r0 & b) continue;
        const int r1 = r0 | b;
        const double2 u = M[r0 + d * col], v = M[r1 + d * col];
        M[r0 + d * col] = cfma(x01, v, cmul(x00, u));
        M[r1 + d * col] = cfma(x11, v, cmul(x10, u));
      }
  }
}

}  // namespace mb
