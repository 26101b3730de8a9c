// Kernels of the family CubicAffine<6> (fused/unfused arithmetic x Float64/Float32 factor).
#include "gsb_kernel_impl.cuh"

namespace gsb {
GSB_DEFINE_ENTRY(cubic6, CubicAffineRows<6>)
}  // namespace gsb
