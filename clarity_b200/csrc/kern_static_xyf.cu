// kern_static_xyf.cu -- compile-time specialised pass kernels (static_dispatch.cuh).
#include "static_dispatch.cuh"

namespace clarity {
template bool static_xy_forward<ProWork>(const PlanEntry&, cudaStream_t, const ProWork&, float2*, cudaError_t*);
template bool static_xy_forward<ProPadded>(const PlanEntry&, cudaStream_t, const ProPadded&, float2*, cudaError_t*);
template bool static_xy_forward<ProImage>(const PlanEntry&, cudaStream_t, const ProImage&, float2*, cudaError_t*);
template bool static_xy_forward<ProAccel>(const PlanEntry&, cudaStream_t, const ProAccel&, float2*, cudaError_t*);
}  // namespace clarity
