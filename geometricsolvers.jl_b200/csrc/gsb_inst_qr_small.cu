// Kernels of the plain step with the static QR factor (QRFactorization, Float64): CubicAffine
// at n = 2, 3, 4 and the two test families.
#include "gsb_kernel_impl.cuh"

namespace gsb {
GSB_DEFINE_QR(cubic2, CubicAffine<2>)
GSB_DEFINE_QR(cubic3, CubicAffine<3>)
GSB_DEFINE_QR(cubic4, CubicAffine<4>)
GSB_DEFINE_QR(hetero6, Hetero6)
GSB_DEFINE_QR(coupled2, Coupled2)
}  // namespace gsb
