// Warp-form kernels of the cubic-affine family at n = 24 with one matrix A for the batch
// (BatchParams: A staged once per CTA, b per system).
#include "gsb_kernel_impl.cuh"

namespace gsb {
KernelEntry* warp_cubic24s(bool fused, bool mixed, bool refine, int T) {
    return pick_warp<WarpCubic<24, true>, 32>(fused, mixed, refine);
}
}  // namespace gsb
