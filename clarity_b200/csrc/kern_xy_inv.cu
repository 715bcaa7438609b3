// kern_xy_inv.cu -- explicit instantiations of the fused pass kernels (see launch.cuh).
#include "launch.cuh"

namespace clarity {
template Status xy_inverse<EpiClip>(Context&, const PlanEntry&, const EpiClip&, const float2*);
template Status xy_inverse<EpiWork>(Context&, const PlanEntry&, const EpiWork&, const float2*);
}  // namespace clarity
