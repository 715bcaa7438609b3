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
#define CLARITY_DYN_SMEM(T, name) T* name = ::clarity_emu::dynamic_smem<T>()
#define CLARITY_BLOCK_STRIDE(n) ((int)blockDim.x)
#define CLARITY_ISSUE_LANES ((int)blockDim.x)
#endif
