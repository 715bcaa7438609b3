// kern_xy_inv2.cu -- explicit instantiations of the fused pass kernels (see launch.cuh).
#include "launch.cuh"

namespace clarity {
template Status xy_inverse<EpiRLProduct>(Context&, const PlanEntry&, const EpiRLProduct&, const float2*);
template Status xy_inverse<MidRLRatio>(Context&, const PlanEntry&, const MidRLRatio&, const float2*);
template Status xy_inverse<EpiJVC>(Context&, const PlanEntry&, const EpiJVC&, const float2*);
}  // namespace clarity
