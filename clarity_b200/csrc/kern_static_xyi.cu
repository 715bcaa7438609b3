// kern_static_xyi.cu -- compile-time specialised pass kernels (static_dispatch.cuh).
#include "static_dispatch.cuh"

namespace clarity {
template bool static_xy_inverse<EpiClip>(const PlanEntry&, cudaStream_t, const EpiClip&, const float2*, cudaError_t*);
template bool static_xy_inverse<EpiWork>(const PlanEntry&, cudaStream_t, const EpiWork&, const float2*, cudaError_t*);
template bool static_xy_inverse<EpiRLProduct>(const PlanEntry&, cudaStream_t, const EpiRLProduct&, const float2*, cudaError_t*);
template bool static_xy_inverse<MidRLRatio>(const PlanEntry&, cudaStream_t, const MidRLRatio&, const float2*, cudaError_t*);
template bool static_xy_inverse<EpiJVC>(const PlanEntry&, cudaStream_t, const EpiJVC&, const float2*, cudaError_t*);
}  // namespace clarity
