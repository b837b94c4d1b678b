// dmb_local.cu -- per-RWG near-block local-inverse preconditioner and its
// learned correction (no counterpart in the reference).
#include "dmb_device.cuh"
#include "dmb_internal.h"

namespace dmb {
void local_inverse_build(dmb_ctx *c, double radius, int kmax) {
  (void)c;
  (void)radius;
  (void)kmax;
  throw DmbError{DMB_ERR_STATE, "local-inverse preconditioner is not available in this build"};
}
}  // namespace dmb
