// emu_cuda.hpp -- TEST INFRASTRUCTURE: host emulation of the few CUDA device
// facilities the library's kernels use, so the kernel sources compile as
// plain C++ (g++, CLARITY_HOST_EMULATION) and run on the CPU under
// AddressSanitizer.  Each block runs on one host thread with blockDim.x == 1:
// every phase's strided loop then covers all its work items and
// __syncthreads is a no-op, which preserves the kernels' semantics.
// Dynamic shared memory is a fresh heap buffer per block, filled with NaN
// bytes so reads of unwritten shared memory poison the result.
#pragma once
#include <cuda_runtime.h>

#include <cmath>
#include <cstdlib>
#include <cstring>

namespace clarity_emu {
extern thread_local uint3 tIdx, bIdx;
extern thread_local dim3 bDim, gDim;
extern thread_local void* smem_ptr;

template <class T>
T* dynamic_smem() {
  return static_cast<T*>(smem_ptr);
}

struct Launcher {
  dim3 grid;
  size_t smem;
  template <class K>
  auto operator()(K kernel) const {
    const dim3 g = grid;
    const size_t s = smem;
    return [g, s, kernel](auto... args) {
      // EMU_BLOCK_ORDER=reverse runs the blocks last to first: a kernel whose
      // result depends on the order of its blocks has an inter-block race
      static const bool reverse = [] {
        const char* v = std::getenv("EMU_BLOCK_ORDER");
        return v && v[0] == 'r';
      }();
      const unsigned long long nb = (unsigned long long)g.x * g.y * g.z;
      for (unsigned long long q = 0; q < nb; ++q) {
        const unsigned long long b = reverse ? nb - 1 - q : q;
        const unsigned bx = (unsigned)(b % g.x), by = (unsigned)((b / g.x) % g.y),
                       bz = (unsigned)(b / ((unsigned long long)g.x * g.y));
        bIdx = make_uint3(bx, by, bz);
        tIdx = make_uint3(0, 0, 0);
        bDim = dim3(1, 1, 1);
        gDim = g;
        void* p = nullptr;
        if (s) {
          p = std::aligned_alloc(128, (s + 127) / 128 * 128);  // as __align__(128)
          std::memset(p, 0xff, s);
        }
        smem_ptr = p;
        kernel(args...);
        std::free(p);
        smem_ptr = nullptr;
      }
    };
  }
};
inline Launcher launcher(long long grid, size_t smem) {
  return Launcher{dim3((unsigned)grid, 1, 1), smem};
}
inline Launcher launcher(dim3 grid, size_t smem) { return Launcher{grid, smem}; }
}  // namespace clarity_emu

#ifndef __noinline__
#define __noinline__
#endif
#ifndef __launch_bounds__
#define __launch_bounds__(...)
#endif

#define threadIdx ::clarity_emu::tIdx
#define blockIdx ::clarity_emu::bIdx
#define blockDim ::clarity_emu::bDim
#define gridDim ::clarity_emu::gDim

template <class T>
inline T __ldg(const T* p) {
  return *p;
}
// A single lane per warp: partners contribute nothing to a sum.
inline float __shfl_xor_sync(unsigned, float, int) { return 0.f; }
inline double __shfl_xor_sync(unsigned, double, int) { return 0.0; }
inline void __syncthreads() {}
// float -> int with truncation (callers keep |x| < 2^31)
inline int __float2int_rz(float x) { return (int)x; }
// blocks run one after another: fences order nothing further, and L2 reads
// are plain reads
inline void __threadfence() {}
template <class T>
inline T __ldcg(const T* p) {
  return *p;
}
// one thread per block: atomics are plain read-modify-writes
inline int atomicAdd(int* p, int v) {
  const int o = *p;
  *p = o + v;
  return o;
}
inline unsigned atomicAdd(unsigned* p, unsigned v) {
  const unsigned o = *p;
  *p = o + v;
  return o;
}
inline float atomicAdd(float* p, float v) {
  const float o = *p;
  *p = o + v;
  return o;
}
inline double atomicAdd(double* p, double v) {
  const double o = *p;
  *p = o + v;
  return o;
}
inline void __syncwarp(unsigned = 0xffffffffu) {}
inline void sincospi(double x, double* s, double* c) {
  *s = std::sin(M_PI * x);
  *c = std::cos(M_PI * x);
}
