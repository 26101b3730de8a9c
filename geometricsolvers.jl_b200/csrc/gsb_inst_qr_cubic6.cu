// Kernels of the plain step with the static QR factor (QRFactorization, Float64): CubicAffine<6>.
#include "gsb_kernel_impl.cuh"

namespace gsb {
GSB_DEFINE_QR(cubic6, CubicAffine<6>)
}  // namespace gsb
