// Kernels of the Float64 LU step with factor reuse or with DogLeg: CubicAffine n = 2, 3, 4 and the
// test families of the reference's batch tests.
#include "gsb_kernel_impl.cuh"

namespace gsb {
GSB_DEFINE_KIND(cubic2, CubicAffineRows<2>)
GSB_DEFINE_KIND(cubic3, CubicAffine<3>)
GSB_DEFINE_KIND(cubic4, CubicAffineRows<4>)
GSB_DEFINE_KIND(hetero6, Hetero6)
GSB_DEFINE_KIND(coupled2, Coupled2)
}  // namespace gsb
