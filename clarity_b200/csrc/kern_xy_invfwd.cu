// kern_xy_invfwd.cu -- explicit instantiations of the fused pass kernels (see launch.cuh).
#include "launch.cuh"

namespace clarity {
template Status xy_inv_fwd<MidRLRatio>(Context&, const PlanEntry&, const MidRLRatio&, float2*);
template Status xy_inv_fwd<EpiJVC>(Context&, const PlanEntry&, const EpiJVC&, float2*);
template Status xy_inv_fwd<EpiRLProduct>(Context&, const PlanEntry&, const EpiRLProduct&, float2*);
template Status xy_inv_fwd<EpiWork>(Context&, const PlanEntry&, const EpiWork&, float2*);
}  // namespace clarity
