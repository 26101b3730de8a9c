// Instantiation: the Levenberg–Marquardt batch kernels of the exponential-sum fit (M = 64).
#include "gsb_kernel_impl.cuh"

namespace gsb {
KernelEntry* lm_expsum3_64(bool fused) {
    return fused ? lm_entry<ExpSum3<64>, true>() : lm_entry<ExpSum3<64>, false>();
}
}  // namespace gsb
