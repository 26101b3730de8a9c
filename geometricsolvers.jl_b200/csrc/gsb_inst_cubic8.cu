// Kernels of the family CubicAffine<8> (fused/unfused arithmetic x Float64/Float32 factor).
#include "gsb_kernel_impl.cuh"

namespace gsb {
GSB_DEFINE_ENTRY(cubic8, CubicAffine<8>)
}  // namespace gsb
