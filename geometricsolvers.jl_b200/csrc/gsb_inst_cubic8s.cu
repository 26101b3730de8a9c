// Kernels of the BatchParams form of CubicAffine<8>: the matrix A shared by the batch (staged
// once per CTA), the right-hand side b per system.
#include "gsb_kernel_impl.cuh"

namespace gsb {
GSB_DEFINE_ENTRY(cubic8s, CubicAffineSharedA<8>)
}  // namespace gsb
