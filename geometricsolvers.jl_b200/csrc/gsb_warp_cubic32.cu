// Warp-form kernels of the cubic-affine family at n = 32 (32 lanes per system).
#include "gsb_kernel_impl.cuh"

namespace gsb {
KernelEntry* warp_cubic32(bool fused, bool mixed, bool refine, int) {
    return pick_warp<WarpCubic<32>, 32>(fused, mixed, refine);
}
}  // namespace gsb
