// launch_macro.cuh -- kernel launch and dynamic shared memory spelled so the
// same sources also compile as host code for the CPU emulation tests
// (tests/emu, CLARITY_HOST_EMULATION): there every block runs on one host
// thread with blockDim.x == 1, and each phase's strided loop covers all of
// its work items, which checks index arithmetic and numerics without a GPU.
#pragma once

#ifndef CLARITY_HOST_EMULATION
#include <cuda_runtime.h>
#define CLARITY_LAUNCH(kernel, grid, block, smem, stream) \
  kernel<<<(grid), (block), (smem), (stream)>>>
namespace clarity {
// Launch with programmatic stream serialisation when pdl is set: the grid may
// be scheduled while the previous kernel on the stream drains its last
// blocks, and every such kernel calls pdl_wait() before it touches memory,
// which returns once the previous grid has completed and its writes are
// visible.  Without pdl this is an ordinary launch.
template <class... P>
struct PdlLauncher {
  void (*k)(P...);
  dim3 grid, block;
  size_t smem;
  cudaStream_t st;
  bool pdl;
  template <class... A>
  void operator()(A&&... args) const {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = pdl ? 1 : 0;
    (void)cudaLaunchKernelEx(&cfg, k, static_cast<A&&>(args)...);
  }
};
template <class... P>
inline PdlLauncher<P...> pdl_launcher(void (*k)(P...), dim3 grid, dim3 block, size_t smem,
                                      cudaStream_t st, bool pdl) {
  return PdlLauncher<P...>{k, grid, block, smem, st, pdl};
}
}  // namespace clarity
#define CLARITY_LAUNCH_PDL(kernel, grid, block, smem, stream, pdl) \
  ::clarity::pdl_launcher((kernel), dim3(grid), dim3(block), (smem), (stream), (pdl))
// First statement of a kernel launched by CLARITY_LAUNCH_PDL.
#define CLARITY_PDL_WAIT() asm volatile("griddepcontrol.wait;" ::: "memory")
#define CLARITY_DYN_SMEM(T, name) extern __shared__ __align__(128) T name[]
// Loop stride of a block-wide strided loop in kernels launched with a
// compile-time block size.
#define CLARITY_BLOCK_STRIDE(n) (n)
// Lanes of the warp that issues bulk copies.
#define CLARITY_ISSUE_LANES 32
#else
#include "emu_cuda.hpp"
#define CLARITY_LAUNCH(kernel, grid, block, smem, stream) \
  ::clarity_emu::launcher((grid), (smem))(kernel)
#define CLARITY_LAUNCH_PDL(kernel, grid, block, smem, stream, pdl) \
  ::clarity_emu::launcher((grid), (smem))(kernel)
#define CLARITY_PDL_WAIT() ((void)0)
#define CLARITY_DYN_SMEM(T, name) T* name = ::clarity_emu::dynamic_smem<T>()
#define CLARITY_BLOCK_STRIDE(n) ((int)blockDim.x)
#define CLARITY_ISSUE_LANES ((int)blockDim.x)
#endif

// The block index and grid size the pass bodies and the operations fused into
// them see, and the qualifier and load they use for their inputs.  A
// translation unit may define these before it includes the passes: the
// persistent batched kernel (kern_batch.cu) runs many work items in one
// block, so an item's tile stands in for the block and the item's pass for
// the grid, and it reads data written earlier in the same launch, which
// needs ordinary coherent loads (no read-only cache, no __restrict__).
#ifndef CLARITY_BLOCK_ID
#define CLARITY_BLOCK_ID() blockIdx.x
#endif
#ifndef CLARITY_GRID_DIM
#define CLARITY_GRID_DIM() gridDim.x
#endif
#ifndef CLARITY_RESTRICT
#define CLARITY_RESTRICT __restrict__
#endif
#ifndef CLARITY_LDG
#define CLARITY_LDG(p) __ldg(p)
#endif
