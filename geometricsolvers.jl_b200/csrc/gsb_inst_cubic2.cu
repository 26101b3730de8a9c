// Kernels of the family CubicAffine<2> (fused/unfused arithmetic x Float64/Float32 factor).
#include "gsb_kernel_impl.cuh"

namespace gsb {
GSB_DEFINE_ENTRY(cubic2, CubicAffineRows<2>)
}  // namespace gsb
