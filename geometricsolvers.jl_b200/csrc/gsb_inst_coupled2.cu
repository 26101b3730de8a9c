// Kernels of the family Coupled2 (fused/unfused arithmetic x Float64/Float32 factor).
#include "gsb_kernel_impl.cuh"

namespace gsb {
GSB_DEFINE_ENTRY(coupled2, Coupled2)
}  // namespace gsb
