// Warp-form kernels of the cubic-affine family at n = 24 (32 lanes per system).
#include "gsb_kernel_impl.cuh"

namespace gsb {
KernelEntry* warp_cubic24(bool fused, bool mixed, bool refine, int) {
    return pick_warp<WarpCubic<24>, 32>(fused, mixed, refine);
}
}  // namespace gsb
