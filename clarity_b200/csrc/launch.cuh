// launch.cuh -- host-side launch wrappers of the fused pass kernels.  The
// template bodies live here; each kern_*.cu file instantiates one family so
// the heavy kernels compile in parallel, and engine.cu sees them through the
// extern declarations at the bottom.
#pragma once
#include "engine.hpp"
#include "ops.cuh"
#include "passes.cuh"

namespace clarity {

// Compile-time specialised launches (static_dispatch.cuh, instantiated in
// kern_static_*.cu).  Each returns true when it launched (error in *err).
template <class F>
bool static_xy_forward(const PlanEntry&, cudaStream_t, const F&, float2*, cudaError_t*);
template <class F>
bool static_z(const PlanEntry&, cudaStream_t, const F&, const float2*, float2*, cudaError_t*);
template <class F>
bool static_xy_inv_fwd(const PlanEntry&, cudaStream_t, const F&, float2*, cudaError_t*);
template <class F>
bool static_xy_inverse(const PlanEntry&, cudaStream_t, const F&, const float2*, cudaError_t*);

#ifndef CL_CHECK
#define CL_CHECK(call)                                         \
  do {                                                         \
    cudaError_t e_ = (call);                                   \
    if (e_ != cudaSuccess) return status_from_cuda(e_, #call); \
  } while (0)
#endif

template <class K>
static cudaError_t prep_kernel(K kernel, int smem) {
  // Opt in to the dynamic shared memory this launch needs (once per kernel).
  return smem_opt_in(reinterpret_cast<const void*>(kernel), smem);
}

template <class Pro>
Status xy_forward(Context& ctx, const PlanEntry& pe, const Pro& pro,
                         float2* S) {
  const VolPlan& P = pe.P;
  cudaError_t se = cudaSuccess;
  if (static_xy_forward(pe, ctx.exec_stream(), pro, S, &se))
    return status_from_cuda(se, "xy forward");
  auto k = k_xy_forward<Pro>;
  CL_CHECK(prep_kernel(k, P.xy_smem));
  note_launch_begin(KK_XY_FORWARD, ctx.exec_stream());
  CLARITY_LAUNCH(k, P.xy_blocks, P.xy_threads, P.xy_smem, ctx.exec_stream())(P, pro, S, pe.tw,
                                                                 pe.xrev);
  note_launch_end(KK_XY_FORWARD, ctx.exec_stream());
  CL_CHECK(cudaGetLastError());
  return Status::Ok();
}

template <class Epi>
Status xy_inverse(Context& ctx, const PlanEntry& pe, const Epi& epi,
                         const float2* S) {
  const VolPlan& P = pe.P;
  cudaError_t se = cudaSuccess;
  if (static_xy_inverse(pe, ctx.exec_stream(), epi, S, &se))
    return status_from_cuda(se, "xy inverse");
  auto k = k_xy_inverse<Epi>;
  CL_CHECK(prep_kernel(k, P.xy_smem));
  note_launch_begin(KK_XY_INVERSE, ctx.exec_stream());
  CLARITY_LAUNCH(k, P.xy_blocks, P.xy_threads, P.xy_smem, ctx.exec_stream())(P, epi, S, pe.tw,
                                                                 pe.xrev);
  note_launch_end(KK_XY_INVERSE, ctx.exec_stream());
  CL_CHECK(cudaGetLastError());
  return Status::Ok();
}

template <class Mid>
Status xy_inv_fwd(Context& ctx, const PlanEntry& pe, const Mid& mid,
                         float2* S) {
  const VolPlan& P = pe.P;
  cudaError_t se = cudaSuccess;
  if (static_xy_inv_fwd(pe, ctx.exec_stream(), mid, S, &se))
    return status_from_cuda(se, "xy inverse+forward");
  auto k = k_xy_inv_fwd<Mid>;
  CL_CHECK(prep_kernel(k, P.xy_smem));
  note_launch_begin(family_of<Mid, KK_XY_INV_FWD>(), ctx.exec_stream());
  CLARITY_LAUNCH(k, P.xy_blocks, P.xy_threads, P.xy_smem, ctx.exec_stream())(P, mid, S, pe.tw,
                                                                 pe.xrev);
  note_launch_end(family_of<Mid, KK_XY_INV_FWD>(), ctx.exec_stream());
  CL_CHECK(cudaGetLastError());
  return Status::Ok();
}

template <class Mod>
Status z_pass(Context& ctx, const PlanEntry& pe, const Mod& mod,
                     const float2* Sin, float2* Sout) {
  const VolPlan& P = pe.P;
  cudaError_t se = cudaSuccess;
  if (static_z(pe, ctx.exec_stream(), mod, Sin, Sout, &se))
    return status_from_cuda(se, "z pass");
  auto k = k_z<Mod>;
  CL_CHECK(prep_kernel(k, P.z_smem));
  note_launch_begin(KK_Z, ctx.exec_stream());
  CLARITY_LAUNCH(k, P.z_blocks, P.z_threads, P.z_smem, ctx.exec_stream())(P, mod, Sin, Sout,
                                                              pe.tw);
  note_launch_end(KK_Z, ctx.exec_stream());
  CL_CHECK(cudaGetLastError());
  return Status::Ok();
}


#define CLARITY_EXTERN_LAUNCHES                                                     \
  extern template Status xy_forward<ProWork>(Context&, const PlanEntry&,            \
                                             const ProWork&, float2*);              \
  extern template Status xy_forward<ProPadded>(Context&, const PlanEntry&,          \
                                               const ProPadded&, float2*);          \
  extern template Status xy_forward<ProImage>(Context&, const PlanEntry&,           \
                                              const ProImage&, float2*);            \
  extern template Status xy_forward<ProAccel>(Context&, const PlanEntry&,           \
                                              const ProAccel&, float2*);            \
  extern template Status xy_inverse<EpiClip>(Context&, const PlanEntry&,            \
                                             const EpiClip&, const float2*);        \
  extern template Status xy_inverse<EpiWork>(Context&, const PlanEntry&,            \
                                             const EpiWork&, const float2*);        \
  extern template Status xy_inverse<EpiRLProduct>(Context&, const PlanEntry&,       \
                                                  const EpiRLProduct&, const float2*); \
  extern template Status xy_inverse<EpiJVC>(Context&, const PlanEntry&,             \
                                            const EpiJVC&, const float2*);          \
  extern template Status xy_inverse<MidRLRatio>(Context&, const PlanEntry&,         \
                                                const MidRLRatio&, const float2*);  \
  extern template Status xy_inv_fwd<MidRLRatio>(Context&, const PlanEntry&,         \
                                                const MidRLRatio&, float2*);        \
  extern template Status xy_inv_fwd<EpiJVC>(Context&, const PlanEntry&,             \
                                            const EpiJVC&, float2*);                \
  extern template Status xy_inv_fwd<EpiRLProduct>(Context&, const PlanEntry&,       \
                                                  const EpiRLProduct&, float2*);    \
  extern template Status xy_inv_fwd<EpiWork>(Context&, const PlanEntry&,            \
                                             const EpiWork&, float2*);              \
  extern template Status z_pass<ModOTF>(Context&, const PlanEntry&, const ModOTF&,  \
                                        const float2*, float2*);                    \
  extern template Status z_pass<ModWiener>(Context&, const PlanEntry&,              \
                                           const ModWiener&, const float2*, float2*); \
  extern template Status z_pass<ModForward>(Context&, const PlanEntry&,             \
                                            const ModForward&, const float2*, float2*);

}  // namespace clarity
