// Warp-form kernels of the cubic-affine family at n = 12 (16 or 32 lanes per system).
#include "gsb_kernel_impl.cuh"

namespace gsb {
KernelEntry* warp_cubic12(bool fused, bool mixed, bool refine, int T) {
    if (T == 32) return pick_warp<WarpCubic<12>, 32>(fused, mixed, refine);
    return pick_warp<WarpCubic<12>, 16>(fused, mixed, refine);
}
}  // namespace gsb
