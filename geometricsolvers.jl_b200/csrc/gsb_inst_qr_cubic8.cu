// Kernels of the plain step with the static QR factor (QRFactorization, Float64): CubicAffine<8>.
#include "gsb_kernel_impl.cuh"

namespace gsb {
GSB_DEFINE_QR(cubic8, CubicAffine<8>)
}  // namespace gsb
