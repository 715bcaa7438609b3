// kern_static_xyif.cu -- compile-time specialised pass kernels (static_dispatch.cuh).
#include "static_dispatch.cuh"

namespace clarity {
template bool static_xy_inv_fwd<MidRLRatio>(const PlanEntry&, cudaStream_t, const MidRLRatio&, float2*, cudaError_t*);
template bool static_xy_inv_fwd<EpiJVC>(const PlanEntry&, cudaStream_t, const EpiJVC&, float2*, cudaError_t*);
template bool static_xy_inv_fwd<EpiRLProduct>(const PlanEntry&, cudaStream_t, const EpiRLProduct&, float2*, cudaError_t*);
template bool static_xy_inv_fwd<EpiWork>(const PlanEntry&, cudaStream_t, const EpiWork&, float2*, cudaError_t*);
}  // namespace clarity
