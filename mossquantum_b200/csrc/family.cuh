// Matrices of the parametric gate families and their binding into a sample's matrix table
// (host and device): k_bind runs bind_record per (record, sample); the host-side lowering
// check runs the same code to bind a circuit on the CPU.
#pragma once
#include <cmath>

#include "kernels.h"

namespace mb {

// Own-order matrix (column-major, m[r + c*d]) of a parametric family at angle t, and its
// derivative generator D = (dU/dt)' U (src/quantum_circuits/gates/differentiation.jl).
// derivative generator D = (dU/dt)' U (src/quantum_circuits/gates/differentiation.jl).
__host__ __device__ inline void family_matrix(int fam, double t, double2* m, double2* g) {
  double s, c;
  sincos(0.5 * t, &s, &c);
  for (int e = 0; e < 64; ++e) { m[e] = cz(); g[e] = cz(); }
  // 2x2 target block u and its generator gu (column-major)
  double2 u[4], gu[4];
  int tfam = fam;
  if (fam >= MB_FAM_CRX && fam <= MB_FAM_CPHASE) tfam = fam - MB_FAM_CRX + MB_FAM_RX;
  if (fam == MB_FAM_CCPHASE) tfam = MB_FAM_PHASE;
  switch (tfam) {
    case MB_FAM_RX:
      u[0] = make_double2(c, 0); u[1] = make_double2(0, -s); u[2] = make_double2(0, -s); u[3] = make_double2(c, 0);
      gu[0] = cz(); gu[1] = make_double2(0, 0.5); gu[2] = make_double2(0, 0.5); gu[3] = cz();
      break;
    case MB_FAM_RY:
      u[0] = make_double2(c, 0); u[1] = make_double2(s, 0); u[2] = make_double2(-s, 0); u[3] = make_double2(c, 0);
      gu[0] = cz(); gu[1] = make_double2(-0.5, 0); gu[2] = make_double2(0.5, 0); gu[3] = cz();
      break;
    case MB_FAM_RZ:
      u[0] = make_double2(c, -s); u[1] = cz(); u[2] = cz(); u[3] = make_double2(c, s);
      gu[0] = make_double2(0, 0.5); gu[1] = cz(); gu[2] = cz(); gu[3] = make_double2(0, -0.5);
      break;
    default: {  // PHASE
      double sp, cp;
      sincos(t, &sp, &cp);
      u[0] = make_double2(1, 0); u[1] = cz(); u[2] = cz(); u[3] = make_double2(cp, sp);
      gu[0] = cz(); gu[1] = cz(); gu[2] = cz(); gu[3] = make_double2(0, -1);
    }
  }
  if (fam <= MB_FAM_PHASE) {
    for (int e = 0; e < 4; ++e) { m[e] = u[e]; g[e] = gu[e]; }
  } else if (fam <= MB_FAM_CPHASE) {
    // CONTROL(u): local bit 0 = control, bit 1 = target; index = control + 2*target.
    m[0 + 0 * 4] = make_double2(1, 0);
    m[2 + 2 * 4] = make_double2(1, 0);
    for (int tr = 0; tr < 2; ++tr)
      for (int tc = 0; tc < 2; ++tc) {
        m[(1 + 2 * tr) + (1 + 2 * tc) * 4] = u[tr + 2 * tc];
        g[(1 + 2 * tr) + (1 + 2 * tc) * 4] = gu[tr + 2 * tc];
      }
  } else {
    // CONTROLCONTROL(PHASE): controls bits 0,1; target bit 2.
    for (int a = 0; a < 8; ++a) m[a + a * 8] = make_double2(1, 0);
    m[7 + 7 * 8] = u[3];
    g[7 + 7 * 8] = gu[3];
  }
}


// Writes record rc's ordered matrix (and generator) at angle t into one sample's table row
// `out`; row0 is the table's first row, which holds the stored operators of a selection.
__host__ __device__ inline void bind_record(const BindRec& rc, double t, const double2* row0, double2* out) {
  if (rc.family == MB_FAM_SELECT) {
    // Copy stored operator j (ordered form, kept in row 0 after the matrix) into this row.
    const int d2 = 1 << (2 * rc.k);
    int j = int(llrint(t));
    j = j < 0 ? 0 : (j > rc.nopt - 1 ? rc.nopt - 1 : j);
    const double2* src = row0 + rc.mat_off + int64_t(d2) * (1 + j);
    for (int e = 0; e < d2; ++e) out[rc.mat_off + e] = src[e];
    return;
  }
  double2 m[64], g[64];
  family_matrix(rc.family, t, m, g);
  const int d = 1 << rc.k;
  const bool adj = rc.flags & MB_OPF_ADJOINT;
  for (int ap = 0; ap < d; ++ap)
    for (int bp = 0; bp < d; ++bp) {
      const int a = rc.perm[ap], bb = rc.perm[bp];
      // ordered[a', b'] = own[perm a', perm b']; adjoint: conj(own[perm b', perm a'])
      out[rc.mat_off + ap + bp * d] = adj ? cconj(m[bb + a * d]) : m[a + bb * d];
      if (rc.gen_off >= 0) {
        double2 gv = g[a + bb * d];
        out[rc.gen_off + ap + bp * d] = adj ? make_double2(-gv.x, -gv.y) : gv;
      }
    }
}

}  // namespace mb
