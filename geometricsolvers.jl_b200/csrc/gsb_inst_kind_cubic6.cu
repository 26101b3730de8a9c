// Kernels of the Float64 LU step with factor reuse or with DogLeg: CubicAffine n = 6.
#include "gsb_kernel_impl.cuh"

namespace gsb {
GSB_DEFINE_KIND(cubic6, CubicAffineRows<6>)
}  // namespace gsb
