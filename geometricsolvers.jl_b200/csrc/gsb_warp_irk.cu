// Warp-form kernels of the Gauss-3 Hénon–Heiles stage systems (n = 12, 16 or 32 lanes per system).
#include "gsb_kernel_impl.cuh"

namespace gsb {
KernelEntry* warp_irk(bool fused, bool mixed, bool refine, int T) {
    if (T == 32) return pick_warp<WarpIrk, 32>(fused, mixed, refine);
    return pick_warp<WarpIrk, 16>(fused, mixed, refine);
}
}  // namespace gsb
