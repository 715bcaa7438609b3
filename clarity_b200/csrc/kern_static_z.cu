// kern_static_z.cu -- compile-time specialised pass kernels (static_dispatch.cuh).
#include "static_dispatch.cuh"

namespace clarity {
template bool static_z<ModOTF>(const PlanEntry&, cudaStream_t, const ModOTF&, const float2*, float2*, cudaError_t*);
template bool static_z<ModWiener>(const PlanEntry&, cudaStream_t, const ModWiener&, const float2*, float2*, cudaError_t*);
template bool static_z<ModForward>(const PlanEntry&, cudaStream_t, const ModForward&, const float2*, float2*, cudaError_t*);
}  // namespace clarity
