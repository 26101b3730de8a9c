// Team kernels of the cubic-affine family at n = 8 (2, 4 or 8 lanes per system).
#include "gsb_kernel_impl.cuh"

namespace gsb {
KernelEntry* team_cubic8(int T, bool mixed) {
    switch (T) {
    case 2: return pick_team<TeamCubic<8>, 2>(mixed);
    case 4: return pick_team<TeamCubic<8>, 4>(mixed);
    case 8: return pick_team<TeamCubic<8>, 8>(mixed);
    default: return nullptr;
    }
}
}  // namespace gsb
