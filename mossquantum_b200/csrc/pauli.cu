// Pauli-string expectation (filled in by the fused bit-mask kernel).
#include "internal.h"

namespace mb {
int pauli_compile(mb_observable o, const mb_term*, size_t) {
  o->pauli_ok = false;
  return MB_OK;
}
int expect_pauli(mb_observable o, mb_state s) { return expect_keys(o, s); }
}  // namespace mb
