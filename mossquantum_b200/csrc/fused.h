// Fused-pass schedule shared by the host scheduler (fused.cu) and the pass kernels.
#pragma once
#include <cstdint>
#include <vector>

#include "internal.h"

namespace mb {

// Micro-op types executed on amplitudes held in registers.
enum MopType : int16_t {
  MOP_U1 = 0,     // dense 2x2 on register bit r0
  MOP_CTRL = 1,   // 2x2 on register bit r0 where every control bit is 1
  MOP_CTRLX = 2,  // swap on register bit r0 where every control bit is 1 (CNOT, TOFFOLI, X)
  MOP_U2 = 3,     // dense 4x4 on register bits r0 < r1 (local bit 0 = r0)
  MOP_DIAG = 4,   // diagonal on up to 3 bits anywhere: factor of local index a where active
  MOP_CPHASE = 5, // factor off[0] (or a sign flip when r1 = 1) where every selector bit is 1
  MOP_GRAD = 6,   // adjoint sweep: accumulate Re<y|D|delta> over register bits r0 (,r1);
                  // nsel = 1 or 2 bits, active = gradient accumulator index within the pass
  MOP_RROT = 7,   // 2x2 with real entries on register bit r0 (RY, H): the real parts of off[0..3]
  MOP_IROT = 8,   // 2x2 with a real diagonal and an imaginary off-diagonal on r0 (RX): Re off[0],
                  // Re off[3], Im off[2], Im off[1]
  MOP_LIFT = 9,   // real rotation [[c,-s],[s,c]] (c >= 0) on r0 as three shears,
                  // x -= t*y; y += s*x; x -= t*y with off[0] = (-t, s), t = s/(1+c)
  MOP_GRADP = 10, // adjoint sweep: Re<y|D|delta> on register bit r0 for a constant generator of
                  // a rotation family, D = (i/2)X, (i/2)Y, (i/2)Z or diag(0, -i) (r1 = 1..4),
                  // negated when conj = 1 (adjoint gates); active = accumulator index
  MOP_CHAN = 11,  // single-qubit channel on a density matrix whose supermatrix is real with the
                  // population/coherence pattern of depolarizing, damping and dephasing channels:
                  // row bit r0, column bit r1, populations x00' = a x00 + b x11, x11' = e x00 +
                  // f x11, coherences x10' = c x10, x01' = d x01 (real parts of off[0..5] = a..f)
};

// Matrix offsets with this bit set index the schedule's own table of derived coefficients
// (rotations and phases of decomposed gates, merged phases) instead of the circuit's table.
constexpr int32_t kXtabFlag = 1 << 29;

// A selector names one index bit: values < 64 are bits of the pass-local amplitude index,
// values >= 64 are bit (sel - 64) of the tile's global base index (constant per tile).
struct MOp {
  int16_t type, r0, r1, nsel;
  int16_t sel[4];
  uint32_t active;   // MOP_DIAG: local indices whose factor is applied
  int16_t conj;      // read the matrix conjugated (density-matrix column pass)
  int16_t param;     // per-sample matrix row (parametric gate with per-sample theta)
  int16_t only;      // reverse sweeps: 0 both states, 1 y only, 2 delta only
  int32_t off[16];   // matrix elements (double2 offsets in a sample's matrix table)
};

constexpr int kMaxRegBits = 5;
struct StageDesc {
  int op0, nops;
  int nreg;
  int reg[kMaxRegBits];  // pass-local bit of register bit k
  int ntid;
  int tid[26];           // pass-local bit of thread-index bit b
};

// TMA box geometry of a tile pass over the amplitude tensor.
struct TmaGeom {
  int ndims;
  int start[5];    // first amplitude bit of the dimension (batch dim: -1)
  int bits[5];     // amplitude bits spanned by the dimension's extent
  int boxb[5];     // amplitude bits covered by the box (tile bits of this dimension)
};

enum PassKind { PASS_TILE = 0, PASS_REG = 1, PASS_PLAIN = 2 };

struct FOp;  // fused.cu

struct Pass {
  int kind;
  int t;                        // tile bits (PASS_TILE) or register bits (PASS_REG)
  std::vector<int> bits;        // pass-local bit i -> global amplitude bit
  std::vector<StageDesc> stages;
  std::vector<MOp> mops;
  std::vector<int> fop_order;   // the schedule's fused ops in the order this pass applies them
  int plain_fop = -1;           // PASS_PLAIN: index into the schedule's fused ops
  bool has_u2 = false;          // holds a 4x4 micro-op (selects the kernel variant)
  void* jit_fn = nullptr;       // specialised kernel (CUfunction) when the JIT is in use
  int ctas = 0;                 // specialised tile kernels: CTAs per SM they were compiled for
  std::vector<int> grad_slots;  // adjoint passes: parameter slot of each gradient accumulator
  int grad_off = 0;             // offset of grad_slots in the schedule's device slot array
  TmaGeom geom{};
  int stage_off = 0, mop_off = 0;  // offsets into the schedule's device buffers
};

}  // namespace mb
