// kern_z.cu -- explicit instantiations of the fused pass kernels (see launch.cuh).
// The z pass keeps scalar complex adds: measured faster than paired FP32
// adds here (its DFT chains are latency-bound), unlike the XY passes.
#define CLARITY_NO_F32X2 1
#include "launch.cuh"

namespace clarity {
template Status z_pass<ModOTF>(Context&, const PlanEntry&, const ModOTF&, const float2*, float2*);
template Status z_pass<ModWiener>(Context&, const PlanEntry&, const ModWiener&, const float2*, float2*);
template Status z_pass<ModForward>(Context&, const PlanEntry&, const ModForward&, const float2*, float2*);
// the kernels noalloc.cu launches directly (CLARITY_EXTERN_PASS_KERNELS)
template __global__ void k_z<ModForward>(const VolPlan, const ModForward, const float2*, float2*,
                                         const float2*);
template __global__ void k_z<ModOTF>(const VolPlan, const ModOTF, const float2*, float2*,
                                     const float2*);
}  // namespace clarity
