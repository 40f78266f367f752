// Tensor-core (tcgen05) fused kernel-block product.  Placeholder until the sm_100a kernel lands.
#include "common.cuh"
#include "context.h"
#include "kernels.h"

namespace tsvm {
bool kermatmul_tc_supported(int, int) { return false; }
tsvm_status kermatmul_tc(tsvm_context *, const float *, const float *, const float *, int64_t, int,
                         double, const float *, int, float *, int, float *) {
  return TSVM_ERR_UNSUPPORTED;
}
}  // namespace tsvm
