// Kernels of the family CubicAffine<4> (fused/unfused arithmetic x Float64/Float32 factor).
#include "gsb_kernel_impl.cuh"

namespace gsb {
GSB_DEFINE_ENTRY(cubic4, CubicAffineRows<4>)
}  // namespace gsb
