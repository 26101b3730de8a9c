// Team kernels of the cubic-affine family at n = 6 (2 lanes per system).
#include "gsb_kernel_impl.cuh"

namespace gsb {
KernelEntry* team_cubic6(int T, bool mixed) {
    switch (T) {
    case 2: return pick_team<TeamCubic<6>, 2>(mixed);
    default: return nullptr;
    }
}
}  // namespace gsb
