// kern_xy_fwd.cu -- explicit instantiations of the fused pass kernels (see launch.cuh).
#include "launch.cuh"

namespace clarity {
template Status xy_forward<ProWork>(Context&, const PlanEntry&, const ProWork&, float2*);
template Status xy_forward<ProPadded>(Context&, const PlanEntry&, const ProPadded&, float2*);
template Status xy_forward<ProImage>(Context&, const PlanEntry&, const ProImage&, float2*);
template Status xy_forward<ProAccel>(Context&, const PlanEntry&, const ProAccel&, float2*);
// the kernels noalloc.cu launches directly (CLARITY_EXTERN_PASS_KERNELS)
template __global__ void k_xy_forward<ProPadded>(const VolPlan, const ProPadded, float2*,
                                                 const float2*, const int*);
template __global__ void k_xy_forward<ProImage>(const VolPlan, const ProImage, float2*,
                                                const float2*, const int*);
}  // namespace clarity
