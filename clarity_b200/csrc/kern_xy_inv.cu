// kern_xy_inv.cu -- explicit instantiations of the fused pass kernels (see launch.cuh).
#include "launch.cuh"

namespace clarity {
template Status xy_inverse<EpiClip>(Context&, const PlanEntry&, const EpiClip&, const float2*);
template Status xy_inverse<EpiWork>(Context&, const PlanEntry&, const EpiWork&, const float2*);
// the kernel noalloc.cu launches directly (CLARITY_EXTERN_PASS_KERNELS)
template __global__ void k_xy_inverse<EpiClip>(const VolPlan, EpiClip, const float2*,
                                               const float2*, const int*);
}  // namespace clarity
