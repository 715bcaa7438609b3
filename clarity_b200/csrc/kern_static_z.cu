// kern_static_z.cu -- compile-time specialised pass kernels (static_dispatch.cuh).
// The z pass keeps scalar complex adds: measured faster than paired FP32
// adds here (its DFT chains are latency-bound), unlike the XY passes.
#define CLARITY_NO_F32X2 1
#include "static_dispatch.cuh"

namespace clarity {
template bool static_z<ModOTF>(const PlanEntry&, cudaStream_t, const ModOTF&, const float2*, float2*, cudaError_t*);
template bool static_z<ModWiener>(const PlanEntry&, cudaStream_t, const ModWiener&, const float2*, float2*, cudaError_t*);
template bool static_z<ModForward>(const PlanEntry&, cudaStream_t, const ModForward&, const float2*, float2*, cudaError_t*);
}  // namespace clarity
