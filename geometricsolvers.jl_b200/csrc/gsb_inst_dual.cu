// Kernels of the families given by their residual alone (the Jacobian from the device dual pass):
// Wood's function with its coupling weight, and the cubic-affine family at n = 2, 3, 4.
#include "gsb_kernel_impl.cuh"

namespace gsb {
GSB_DEFINE_ENTRY(wood, DualFamily<WoodFn>)
GSB_DEFINE_ENTRY(cubicdual2, DualFamily<CubicAffineFn<2>>)
GSB_DEFINE_ENTRY(cubicdual3, DualFamily<CubicAffineFn<3>>)
GSB_DEFINE_ENTRY(cubicdual4, DualFamily<CubicAffineFn<4>>)
}  // namespace gsb
