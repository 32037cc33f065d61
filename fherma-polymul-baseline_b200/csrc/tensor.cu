// Tensor-core residue conversion and CRT (tcgen05 kind::i8) -- placeholder
// until the INT8 contraction kernels land; plans asking for it are refused.
#include "pm_internal.h"
#include "../../include/polymul.h"

namespace pm {
void tensor_init(PlanCore&) { throw Failure(PM_ERR_UNSUPPORTED, "tensor conversion not available yet"); }
void tensor_release(PlanCore&) {}
void launch_tensor(const PlanCore&, const uint32_t*, const uint32_t*, uint32_t*, uint32_t*, cudaStream_t) {
    throw Failure(PM_ERR_UNSUPPORTED, "tensor conversion not available yet");
}
}  // namespace pm
