// Kernels of the mixed LU step with Float32 line-search trials: CubicAffine n = 2, 3, 4, 6.
#include "gsb_kernel_impl.cuh"

namespace gsb {
GSB_DEFINE_TRIAL32(cubic2, CubicAffineRows<2>)
GSB_DEFINE_TRIAL32(cubic3, CubicAffine<3>)
GSB_DEFINE_TRIAL32(cubic4, CubicAffineRows<4>)
GSB_DEFINE_TRIAL32(cubic6, CubicAffineRows<6>)
}  // namespace gsb
