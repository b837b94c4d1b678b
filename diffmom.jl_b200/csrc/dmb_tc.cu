// dmb_tc.cu -- tensor-core (tcgen05) kernels.  Placeholder until the sm_100a
// 3xTF32 complex update lands: reports no tensor-core path.
#include "dmb_device.cuh"
#include "dmb_internal.h"

namespace dmb {
bool tc_available(dmb_ctx *c) {
  (void)c;
  return false;
}
void tc_ldlt_update_c64(dmb_ctx *c, int64_t N, int64_t j0, int64_t jcol, int b, float2 *F, const float2 *W) {
  (void)c; (void)N; (void)j0; (void)jcol; (void)b; (void)F; (void)W;
  throw DmbError{DMB_ERR_STATE, "tensor-core update not available"};
}
}  // namespace dmb
