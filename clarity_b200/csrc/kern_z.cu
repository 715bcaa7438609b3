// kern_z.cu -- explicit instantiations of the fused pass kernels (see launch.cuh).
#include "launch.cuh"

namespace clarity {
template Status z_pass<ModOTF>(Context&, const PlanEntry&, const ModOTF&, const float2*, float2*);
template Status z_pass<ModWiener>(Context&, const PlanEntry&, const ModWiener&, const float2*, float2*);
template Status z_pass<ModForward>(Context&, const PlanEntry&, const ModForward&, const float2*, float2*);
}  // namespace clarity
