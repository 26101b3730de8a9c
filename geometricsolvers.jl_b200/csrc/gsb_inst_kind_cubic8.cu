// Kernels of the Float64 LU step with factor reuse or with DogLeg: CubicAffine n = 8.
#include "gsb_kernel_impl.cuh"

namespace gsb {
GSB_DEFINE_KIND(cubic8, CubicAffineRows<8>)
}  // namespace gsb
