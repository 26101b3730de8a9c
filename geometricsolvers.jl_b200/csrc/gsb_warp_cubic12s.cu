// Warp-form kernels of the cubic-affine family at n = 12 with one matrix A for the batch
// (BatchParams: A staged once per CTA, b per system).
#include "gsb_kernel_impl.cuh"

namespace gsb {
KernelEntry* warp_cubic12s(bool fused, bool mixed, bool refine, int T) {
    if (T == 32) return pick_warp<WarpCubic<12, true>, 32>(fused, mixed, refine);
    return pick_warp<WarpCubic<12, true>, 16>(fused, mixed, refine);
}
}  // namespace gsb
