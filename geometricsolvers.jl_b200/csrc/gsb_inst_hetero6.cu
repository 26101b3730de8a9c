// Kernels of the family Hetero6 (fused/unfused arithmetic x Float64/Float32 factor).
#include "gsb_kernel_impl.cuh"

namespace gsb {
GSB_DEFINE_ENTRY(hetero6, Hetero6)
}  // namespace gsb
