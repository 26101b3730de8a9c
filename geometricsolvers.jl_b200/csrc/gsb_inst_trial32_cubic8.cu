// Kernels of the mixed LU step with Float32 line-search trials: CubicAffine n = 8.
#include "gsb_kernel_impl.cuh"

namespace gsb {
GSB_DEFINE_TRIAL32(cubic8, CubicAffineRows<8>)
}  // namespace gsb
