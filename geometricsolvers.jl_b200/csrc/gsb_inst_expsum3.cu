// Instantiation: the Levenberg–Marquardt batch kernels of the exponential-sum fit (M = 64): the
// FP64 stacked factor, and the mixed form (FP32 factor, FP64 refinement).
#include "gsb_kernel_impl.cuh"

namespace gsb {
KernelEntry* lm_expsum3_64(bool fused, bool mixed) {
    if (mixed) return fused ? lm_entry<ExpSum3<64>, true, true>() : lm_entry<ExpSum3<64>, false, true>();
    return fused ? lm_entry<ExpSum3<64>, true, false>() : lm_entry<ExpSum3<64>, false, false>();
}
}  // namespace gsb
