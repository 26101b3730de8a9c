// Kernels of the BatchParams form of CubicAffine<4>: the matrix A shared by the batch (staged
// once per CTA), the right-hand side b per system.
#include "gsb_kernel_impl.cuh"

namespace gsb {
GSB_DEFINE_ENTRY(cubic4s, CubicAffineSharedA<4>)
}  // namespace gsb
