// Kernels of the family CubicAffine<3> (fused/unfused arithmetic x Float64/Float32 factor).
#include "gsb_kernel_impl.cuh"

namespace gsb {
GSB_DEFINE_ENTRY(cubic3, CubicAffine<3>)
}  // namespace gsb
