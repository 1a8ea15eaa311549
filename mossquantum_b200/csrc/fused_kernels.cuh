// Device side of the fused passes (K1 TMA tile kernel, K2 register sweep kernel).
//
// Both kernels hold 2^R amplitudes per thread in registers; register bit k of a thread's
// amplitude index j is pass-local bit reg[k]. A stage loads the registers, runs its
// micro-ops and stores them back. Gates on other bits of a tile run in later stages after a
// shared-memory exchange; diagonal gates and controls read any index bit directly.
#pragma once
#include <cuda.h>

#include "fused.h"

namespace mb {
namespace fk {

// Matrix element at `off`: the circuit's table row m, or the schedule's derived table x when
// the offset carries kXtabFlag.
__device__ __forceinline__ double2 ldm(const double2* m, const double2* x, int off, int conj) {
  const double2 v = (off & kXtabFlag) ? __ldg(x + (off & ~kXtabFlag)) : __ldg(m + off);
  return conj ? make_double2(v.x, -v.y) : v;
}

// Index bit of amplitude j (j is a compile-time register index).
template <int R>
__device__ __forceinline__ uint64_t reg_offset(int j, const int* reg) {
  uint64_t o = 0;
#pragma unroll
  for (int k = 0; k < R; ++k)
    if ((j >> k) & 1) o |= uint64_t(1) << reg[k];
  return o;
}

// A selector resolved for one thread: the register bit it reads (rk >= 0) or its constant
// value for every amplitude the thread holds (thread-index or tile-base bit).
struct Sel {
  int rk;
  uint32_t cv;
};

template <int R>
__device__ __forceinline__ Sel resolve(int16_t sel, uint64_t lbase, const int* reg, uint64_t gbase) {
  Sel r{-1, 0u};
  if (sel >= 64) {
    r.cv = uint32_t((gbase >> (sel - 64)) & 1);
    return r;
  }
#pragma unroll
  for (int k = 0; k < R; ++k)
    if (reg[k] == sel) r.rk = k;
  if (r.rk < 0) r.cv = uint32_t((lbase >> sel) & 1);
  return r;
}

__device__ __forceinline__ uint32_t sel_val(const Sel& s, int j) {
  return s.rk >= 0 ? uint32_t((j >> s.rk) & 1) : s.cv;
}

template <int R, int K>
__device__ __forceinline__ void u1(double2 (&a)[1 << R], double2 m00, double2 m10, double2 m01, double2 m11) {
#pragma unroll
  for (int j = 0; j < (1 << R); ++j)
    if (!((j >> K) & 1)) {
      const double2 x = a[j], y = a[j | (1 << K)];
      a[j] = cfma(m01, y, cmul(m00, x));
      a[j | (1 << K)] = cfma(m11, y, cmul(m10, x));
    }
}

// Real 2x2 [[a, b], [c, d]] on register bit K: four real multiply-adds per amplitude.
template <int R, int K>
__device__ __forceinline__ void rrot(double2 (&v)[1 << R], double a, double c, double b, double d) {
#pragma unroll
  for (int j = 0; j < (1 << R); ++j)
    if (!((j >> K) & 1)) {
      const double2 x = v[j], y = v[j | (1 << K)];
      v[j] = make_double2(fma(b, y.x, a * x.x), fma(b, y.y, a * x.y));
      v[j | (1 << K)] = make_double2(fma(d, y.x, c * x.x), fma(d, y.y, c * x.y));
    }
}

// [[a, i*b], [i*c, d]] with real a, b, c, d on register bit K.
template <int R, int K>
__device__ __forceinline__ void irot(double2 (&v)[1 << R], double a, double ci, double bi, double d) {
#pragma unroll
  for (int j = 0; j < (1 << R); ++j)
    if (!((j >> K) & 1)) {
      const double2 x = v[j], y = v[j | (1 << K)];
      v[j] = make_double2(fma(-bi, y.y, a * x.x), fma(bi, y.x, a * x.y));
      v[j | (1 << K)] = make_double2(fma(-ci, x.y, d * y.x), fma(ci, x.x, d * y.y));
    }
}

// Rotation by three shears (mt = -t, s): three fused multiply-adds per component and pair.
template <int R, int K>
__device__ __forceinline__ void lift(double2 (&v)[1 << R], double mt, double s) {
#pragma unroll
  for (int j = 0; j < (1 << R); ++j)
    if (!((j >> K) & 1)) {
      double2 x = v[j], y = v[j | (1 << K)];
      x.x = fma(mt, y.x, x.x);
      x.y = fma(mt, y.y, x.y);
      y.x = fma(s, x.x, y.x);
      y.y = fma(s, x.y, y.y);
      x.x = fma(mt, y.x, x.x);
      x.y = fma(mt, y.y, x.y);
      v[j] = x;
      v[j | (1 << K)] = y;
    }
}

template <int R, int K>
__device__ __forceinline__ void ctrl(double2 (&a)[1 << R], double2 m00, double2 m10, double2 m01, double2 m11,
                                     const MOp* __restrict__ op, int nsel, uint64_t lbase, const int* reg,
                                     uint64_t gbase, bool swap_only) {
  // Controls: a mask over register bits that must be set, and a thread-constant condition.
  uint32_t need = 0, cst = 1;
  for (int c = 0; c < nsel; ++c) {
    const Sel sl = resolve<R>(op->sel[c], lbase, reg, gbase);
    if (sl.rk >= 0) need |= 1u << sl.rk;
    else cst &= sl.cv;
  }
  if (!cst) return;
#pragma unroll
  for (int j = 0; j < (1 << R); ++j)
    if (!((j >> K) & 1)) {
      const uint32_t on = (uint32_t(j) & need) == need;
      const double2 x = a[j], y = a[j | (1 << K)];
      double2 nx, ny;
      if (swap_only) {
        nx = y;
        ny = x;
      } else {
        nx = cfma(m01, y, cmul(m00, x));
        ny = cfma(m11, y, cmul(m10, x));
      }
      a[j] = on ? nx : x;
      a[j | (1 << K)] = on ? ny : y;
    }
}

template <int R, int K0, int K1>
__device__ __forceinline__ void u2(double2 (&a)[1 << R], const double2* m, const double2* x, const MOp* __restrict__ op,
                                   int conj) {
  double2 u[16];
#pragma unroll
  for (int e = 0; e < 16; ++e) u[e] = ldm(m, x, op->off[e], conj);
#pragma unroll
  for (int j = 0; j < (1 << R); ++j)
    if (!((j >> K0) & 1) && !((j >> K1) & 1)) {
      const int i0 = j, i1 = j | (1 << K0), i2 = j | (1 << K1), i3 = j | (1 << K0) | (1 << K1);
      const double2 x0 = a[i0], x1 = a[i1], x2 = a[i2], x3 = a[i3];
      a[i0] = cfma(u[12], x3, cfma(u[8], x2, cfma(u[4], x1, cmul(u[0], x0))));
      a[i1] = cfma(u[13], x3, cfma(u[9], x2, cfma(u[5], x1, cmul(u[1], x0))));
      a[i2] = cfma(u[14], x3, cfma(u[10], x2, cfma(u[6], x1, cmul(u[2], x0))));
      a[i3] = cfma(u[15], x3, cfma(u[11], x2, cfma(u[7], x1, cmul(u[3], x0))));
    }
}

// Real channel supermatrix on (row bit K0, column bit K1): populations mix through a 2x2,
// coherences scale (MOP_CHAN).
template <int R, int K0, int K1>
__device__ __forceinline__ void chan(double2 (&a)[1 << R], double ca, double cb, double cc, double cd, double ce,
                                     double cf) {
#pragma unroll
  for (int j = 0; j < (1 << R); ++j)
    if (!((j >> K0) & 1) && !((j >> K1) & 1)) {
      const int i1 = j | (1 << K0), i2 = j | (1 << K1), i3 = j | (1 << K0) | (1 << K1);
      const double2 x0 = a[j], x3 = a[i3];
      a[j] = make_double2(fma(ca, x0.x, cb * x3.x), fma(ca, x0.y, cb * x3.y));
      a[i3] = make_double2(fma(ce, x0.x, cf * x3.x), fma(ce, x0.y, cf * x3.y));
      a[i1] = make_double2(cc * a[i1].x, cc * a[i1].y);
      a[i2] = make_double2(cd * a[i2].x, cd * a[i2].y);
    }
}

template <int R>
__device__ __forceinline__ void diag(double2 (&a)[1 << R], const double2* m, const double2* xt, const MOp* __restrict__ op,
                                     int nsel, int conj, uint64_t lbase, const int* reg, uint64_t gbase) {
  const uint32_t active = op->active;
  Sel sl[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) sl[c] = c < nsel ? resolve<R>(op->sel[c], lbase, reg, gbase) : Sel{-1, 0u};
  double2 f[8];
#pragma unroll
  for (int e = 0; e < 8; ++e)
    f[e] = (e < (1 << nsel) && ((active >> e) & 1)) ? ldm(m, xt, op->off[e], conj) : make_double2(1.0, 0.0);
#pragma unroll
  for (int j = 0; j < (1 << R); ++j) {
    const uint32_t idx = sel_val(sl[0], j) | (sel_val(sl[1], j) << 1) | (sel_val(sl[2], j) << 2);
    if ((active >> idx) & 1) {
      double2 fac = f[0];
#pragma unroll
      for (int e = 1; e < 8; ++e) fac = (idx == uint32_t(e)) ? f[e] : fac;
      a[j] = cmul(fac, a[j]);
    }
  }
}

// Controlled-X with the control mask NEED over register bits known at compile time: the
// swap is a renaming of registers and costs no instructions.
template <int R, int K, int NEED>
__device__ __forceinline__ void ctrlx_ct(double2 (&a)[1 << R]) {
#pragma unroll
  for (int j = 0; j < (1 << R); ++j)
    if (!((j >> K) & 1) && (j & NEED) == NEED) {
      const double2 x = a[j];
      a[j] = a[j | (1 << K)];
      a[j | (1 << K)] = x;
    }
}

template <int R, int K, int NEED = 0>
__device__ __forceinline__ void ctrlx_dispatch(double2 (&a)[1 << R], int need) {
  if constexpr (NEED < (1 << R)) {
    if constexpr (!((NEED >> K) & 1)) {
      if (need == NEED) {
        ctrlx_ct<R, K, NEED>(a);
        return;
      }
    }
    ctrlx_dispatch<R, K, NEED + 1>(a, need);
  }
}

// Phase factor f on the amplitudes whose register bits cover NEED (compile-time mask).
template <int R, int NEED>
__device__ __forceinline__ void cphase_ct(double2 (&a)[1 << R], double2 f, bool neg) {
#pragma unroll
  for (int j = 0; j < (1 << R); ++j)
    if ((j & NEED) == NEED) a[j] = neg ? make_double2(-a[j].x, -a[j].y) : cmul(f, a[j]);
}

template <int R, int NEED = 0>
__device__ __forceinline__ void cphase_dispatch(double2 (&a)[1 << R], int need, double2 f, bool neg) {
  if constexpr (NEED < (1 << R)) {
    if (need == NEED) {
      cphase_ct<R, NEED>(a, f, neg);
      return;
    }
    cphase_dispatch<R, NEED + 1>(a, need, f, neg);
  }
}

#define FK_CASE_K(R, K, CALL) case K: { constexpr int KK = K; if constexpr (KK < R) { CALL; } } break;

// Runs micro-ops [0, nops) on the registers. HAS_U2 = false compiles a lean variant without
// the 4x4 path (fewer live registers) for passes that hold no two-qubit dense gate.
// xt0: the schedule's fixed derived entries; xb: this sample's row of per-sample entries.
template <int R, bool HAS_U2>
__device__ __forceinline__ void run_mops(double2 (&a)[1 << R], const MOp* __restrict__ mops, int nops,
                                         uint64_t lbase, const int* reg, uint64_t gbase,
                                         const double2* __restrict__ tab, const double2* __restrict__ xt0,
                                         const double2* __restrict__ xb, int64_t tstride, int b) {
  for (int q = 0; q < nops; ++q) {
    const MOp* __restrict__ op = mops + q;
    const int type = op->type, r0 = op->r0, nsel = op->nsel, conj = op->conj;
    const double2* m = tab + (op->param ? int64_t(b) * tstride : 0);
    const double2* xt = op->param ? xb : xt0;
    if (type == MOP_LIFT) {
      const double2 ts = ldm(m, xt, op->off[0], 0);
      switch (r0) {
        FK_CASE_K(R, 0, (lift<R, KK>(a, ts.x, ts.y)))
        FK_CASE_K(R, 1, (lift<R, KK>(a, ts.x, ts.y)))
        FK_CASE_K(R, 2, (lift<R, KK>(a, ts.x, ts.y)))
        FK_CASE_K(R, 3, (lift<R, KK>(a, ts.x, ts.y)))
        FK_CASE_K(R, 4, (lift<R, KK>(a, ts.x, ts.y)))
      }
    } else if (type == MOP_RROT || type == MOP_IROT) {
      const double2 m00 = ldm(m, xt, op->off[0], conj), m10 = ldm(m, xt, op->off[1], conj);
      const double2 m01 = ldm(m, xt, op->off[2], conj), m11 = ldm(m, xt, op->off[3], conj);
      if (type == MOP_RROT) {
        switch (r0) {
          FK_CASE_K(R, 0, (rrot<R, KK>(a, m00.x, m10.x, m01.x, m11.x)))
          FK_CASE_K(R, 1, (rrot<R, KK>(a, m00.x, m10.x, m01.x, m11.x)))
          FK_CASE_K(R, 2, (rrot<R, KK>(a, m00.x, m10.x, m01.x, m11.x)))
          FK_CASE_K(R, 3, (rrot<R, KK>(a, m00.x, m10.x, m01.x, m11.x)))
          FK_CASE_K(R, 4, (rrot<R, KK>(a, m00.x, m10.x, m01.x, m11.x)))
        }
      } else {
        switch (r0) {
          FK_CASE_K(R, 0, (irot<R, KK>(a, m00.x, m10.y, m01.y, m11.x)))
          FK_CASE_K(R, 1, (irot<R, KK>(a, m00.x, m10.y, m01.y, m11.x)))
          FK_CASE_K(R, 2, (irot<R, KK>(a, m00.x, m10.y, m01.y, m11.x)))
          FK_CASE_K(R, 3, (irot<R, KK>(a, m00.x, m10.y, m01.y, m11.x)))
          FK_CASE_K(R, 4, (irot<R, KK>(a, m00.x, m10.y, m01.y, m11.x)))
        }
      }
    } else if (type == MOP_U1) {
      const double2 m00 = ldm(m, xt, op->off[0], conj), m10 = ldm(m, xt, op->off[1], conj);
      const double2 m01 = ldm(m, xt, op->off[2], conj), m11 = ldm(m, xt, op->off[3], conj);
      switch (r0) {
        FK_CASE_K(R, 0, (u1<R, KK>(a, m00, m10, m01, m11)))
        FK_CASE_K(R, 1, (u1<R, KK>(a, m00, m10, m01, m11)))
        FK_CASE_K(R, 2, (u1<R, KK>(a, m00, m10, m01, m11)))
        FK_CASE_K(R, 3, (u1<R, KK>(a, m00, m10, m01, m11)))
        FK_CASE_K(R, 4, (u1<R, KK>(a, m00, m10, m01, m11)))
      }
    } else if (type == MOP_CTRLX || type == MOP_CPHASE) {
      // Resolve the selectors: register-bit mask plus a thread-constant condition.
      int need = 0;
      uint32_t cst = 1;
      for (int c = 0; c < nsel; ++c) {
        const Sel sl = resolve<R>(op->sel[c], lbase, reg, gbase);
        if (sl.rk >= 0) need |= 1 << sl.rk;
        else cst &= sl.cv;
      }
      if (cst) {
        if (type == MOP_CTRLX) {
          switch (r0) {
            FK_CASE_K(R, 0, (ctrlx_dispatch<R, KK>(a, need)))
            FK_CASE_K(R, 1, (ctrlx_dispatch<R, KK>(a, need)))
            FK_CASE_K(R, 2, (ctrlx_dispatch<R, KK>(a, need)))
            FK_CASE_K(R, 3, (ctrlx_dispatch<R, KK>(a, need)))
            FK_CASE_K(R, 4, (ctrlx_dispatch<R, KK>(a, need)))
          }
        } else {
          const bool neg = op->r1 != 0;
          const double2 f = neg ? make_double2(-1.0, 0.0) : ldm(m, xt, op->off[0], conj);
          cphase_dispatch<R>(a, need, f, neg);
        }
      }
    } else if (type == MOP_CTRL) {
      const bool sw = false;
      double2 m00 = make_double2(0, 0), m10 = m00, m01 = m00, m11 = m00;
      if (!sw) {
        m00 = ldm(m, xt, op->off[0], conj);
        m10 = ldm(m, xt, op->off[1], conj);
        m01 = ldm(m, xt, op->off[2], conj);
        m11 = ldm(m, xt, op->off[3], conj);
      }
      switch (r0) {
        FK_CASE_K(R, 0, (ctrl<R, KK>(a, m00, m10, m01, m11, op, nsel, lbase, reg, gbase, sw)))
        FK_CASE_K(R, 1, (ctrl<R, KK>(a, m00, m10, m01, m11, op, nsel, lbase, reg, gbase, sw)))
        FK_CASE_K(R, 2, (ctrl<R, KK>(a, m00, m10, m01, m11, op, nsel, lbase, reg, gbase, sw)))
        FK_CASE_K(R, 3, (ctrl<R, KK>(a, m00, m10, m01, m11, op, nsel, lbase, reg, gbase, sw)))
        FK_CASE_K(R, 4, (ctrl<R, KK>(a, m00, m10, m01, m11, op, nsel, lbase, reg, gbase, sw)))
      }
    } else if (type == MOP_DIAG) {
      diag<R>(a, m, xt, op, nsel, conj, lbase, reg, gbase);
    } else if constexpr (HAS_U2) {
      if (type == MOP_CHAN) {
        const double ca = ldm(m, xt, op->off[0], 0).x, cb = ldm(m, xt, op->off[1], 0).x;
        const double cc = ldm(m, xt, op->off[2], 0).x, cd = ldm(m, xt, op->off[3], 0).x;
        const double ce = ldm(m, xt, op->off[4], 0).x, cf = ldm(m, xt, op->off[5], 0).x;
#define FK_CHAN(K0, K1) \
  case K0 * 8 + K1: if constexpr (K0 < R && K1 < R) chan<R, K0, K1>(a, ca, cb, cc, cd, ce, cf); break;
        switch (r0 * 8 + op->r1) {
          FK_CHAN(0, 1) FK_CHAN(0, 2) FK_CHAN(0, 3) FK_CHAN(0, 4) FK_CHAN(1, 0) FK_CHAN(1, 2) FK_CHAN(1, 3)
          FK_CHAN(1, 4) FK_CHAN(2, 0) FK_CHAN(2, 1) FK_CHAN(2, 3) FK_CHAN(2, 4) FK_CHAN(3, 0) FK_CHAN(3, 1)
          FK_CHAN(3, 2) FK_CHAN(3, 4) FK_CHAN(4, 0) FK_CHAN(4, 1) FK_CHAN(4, 2) FK_CHAN(4, 3)
        }
#undef FK_CHAN
      }
      if (type == MOP_U2) {
        switch (r0 * 8 + op->r1) {
          case 0 * 8 + 1: u2<R, 0, 1>(a, m, xt, op, conj); break;
          case 0 * 8 + 2: u2<R, 0, 2>(a, m, xt, op, conj); break;
          case 0 * 8 + 3: u2<R, 0, 3>(a, m, xt, op, conj); break;
          case 1 * 8 + 2: u2<R, 1, 2>(a, m, xt, op, conj); break;
          case 1 * 8 + 3: u2<R, 1, 3>(a, m, xt, op, conj); break;
          case 2 * 8 + 3: u2<R, 2, 3>(a, m, xt, op, conj); break;
          default:
            if constexpr (R > 4) {
              switch (r0 * 8 + op->r1) {
                case 0 * 8 + 4: u2<R, 0, 4>(a, m, xt, op, conj); break;
                case 1 * 8 + 4: u2<R, 1, 4>(a, m, xt, op, conj); break;
                case 2 * 8 + 4: u2<R, 2, 4>(a, m, xt, op, conj); break;
                case 3 * 8 + 4: u2<R, 3, 4>(a, m, xt, op, conj); break;
              }
            }
        }
      }
    }
  }
}

// ---- TMA / mbarrier primitives (plain per-CTA loads and stores, no multicast) -----------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

// Bounded wait on phase `parity`; returns false when the limit ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  const uint32_t addr = smem_u32(bar);
  for (uint32_t it = 0; it < (1u << 26); ++it) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(addr), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void tma_load(const CUtensorMap* map, void* dst, uint64_t* bar, int nd, const int* c) {
  const uint64_t m = reinterpret_cast<uint64_t>(map);
  const uint32_t d = smem_u32(dst), b = smem_u32(bar);
  switch (nd) {
    case 1:
      asm volatile("cp.async.bulk.tensor.1d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2}], [%3];"
                   ::"r"(d), "l"(m), "r"(c[0]), "r"(b) : "memory");
      break;
    case 2:
      asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
                   ::"r"(d), "l"(m), "r"(c[0]), "r"(c[1]), "r"(b) : "memory");
      break;
    case 3:
      asm volatile("cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
                   ::"r"(d), "l"(m), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(b) : "memory");
      break;
    case 4:
      asm volatile("cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];"
                   ::"r"(d), "l"(m), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(c[3]), "r"(b) : "memory");
      break;
    default:
      asm volatile("cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5, %6}], [%7];"
                   ::"r"(d), "l"(m), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(c[3]), "r"(c[4]), "r"(b) : "memory");
  }
}

__device__ __forceinline__ void tma_store(const CUtensorMap* map, const void* src, int nd, const int* c) {
  const uint64_t m = reinterpret_cast<uint64_t>(map);
  const uint32_t s = smem_u32(src);
  switch (nd) {
    case 1:
      asm volatile("cp.async.bulk.tensor.1d.global.shared::cta.tile.bulk_group [%0, {%2}], [%1];"
                   ::"l"(m), "r"(s), "r"(c[0]) : "memory");
      break;
    case 2:
      asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.tile.bulk_group [%0, {%2, %3}], [%1];"
                   ::"l"(m), "r"(s), "r"(c[0]), "r"(c[1]) : "memory");
      break;
    case 3:
      asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.tile.bulk_group [%0, {%2, %3, %4}], [%1];"
                   ::"l"(m), "r"(s), "r"(c[0]), "r"(c[1]), "r"(c[2]) : "memory");
      break;
    case 4:
      asm volatile("cp.async.bulk.tensor.4d.global.shared::cta.tile.bulk_group [%0, {%2, %3, %4, %5}], [%1];"
                   ::"l"(m), "r"(s), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(c[3]) : "memory");
      break;
    default:
      asm volatile("cp.async.bulk.tensor.5d.global.shared::cta.tile.bulk_group [%0, {%2, %3, %4, %5, %6}], [%1];"
                   ::"l"(m), "r"(s), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(c[3]), "r"(c[4]) : "memory");
  }
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}

__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 16-byte slot of tile-local amplitude i under the 128-byte TMA swizzle.
__device__ __forceinline__ uint32_t swz(uint32_t i) { return i ^ ((i >> 3) & 7u); }

}  // namespace fk

struct TileArgs {
  int t;               // tile bits
  int nstages;
  int ndims;
  int start[5];        // TMA dims: first amplitude bit (-1 = batch dimension)
  int extb[5];         // bits spanned by the dimension extent
  int bits[16];        // tile-local bit -> global amplitude bit
  int64_t tiles_per_sample;
  int64_t ntiles;
  int64_t tstride;     // matrix-table row stride for per-sample parameters
  const StageDesc* stages;
  const MOp* mops;
  const double2* table;
  const double2* xtab;     // the schedule's derived coefficients (kXtabFlag offsets)
  const double2* xtabs;    // per-sample derived entries, row b at xtabs + b * xrow
  int64_t xrow;
  unsigned* err;
};

struct RegArgs {
  int nbits;           // register bits
  int reg[kMaxRegBits];  // global bits held in registers (ascending)
  int N;               // amplitude bits of one sample
  int64_t groups;      // per sample: 2^(N - nbits)
  int nsamples;
  int nops;
  int64_t tstride;
  const MOp* mops;
  const double2* table;
  const double2* xtab;
  const double2* xtabs;
  int64_t xrow;
};

}  // namespace mb
