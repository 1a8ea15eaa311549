// Fused-pass execution (filled in by the tiled kernels).
#include "internal.h"

namespace mb {
int apply_fused(mb_circuit c, mb_state s, int64_t mrow_stride) { return apply_plain(c, s, mrow_stride); }
void release_schedules(mb_circuit) {}
}  // namespace mb

extern "C" int mb_circuit_passes(mb_circuit c, int* npasses) {
  if (!c || !npasses) return MB_EINVAL;
  *npasses = int(c->ops.size());
  return MB_OK;
}
