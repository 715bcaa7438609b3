// tma.cuh -- bulk asynchronous copies (TMA, cp.async.bulk) between global
// and shared memory, completed on an mbarrier, for sm_100a.
//
// Only plain one-CTA copies are used: every source is this GPU's own memory
// and no copy is broadcast to other CTAs.  Every address and size is a
// multiple of 16 bytes (the rule for untiled bulk copies); callers check
// that at compile time.  Waits are bounded: after kWaitLimit polls a wait
// records an error code in *err and gives up, so a lost completion can
// never hang the GPU.
#pragma once
#include <cstddef>
#include <cstdint>

#include "launch_macro.cuh"
#ifndef CLARITY_HOST_EMULATION
#include <cuda.h>  // CUtensorMap (the type only; the encoder is fetched at run time)
#endif

namespace clarity {

constexpr long long kWaitLimit = 1ll << 22;  // polls of mbarrier.try_wait
constexpr int kErrWaitTimeout = 1;
constexpr int kErrMisaligned = 2;

#ifndef CLARITY_HOST_EMULATION
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// global -> shared, completes `bytes` of the barrier's transaction count
__device__ __forceinline__ void bulk_load(void* dst_smem, const void* src_gmem,
                                          uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes "
      "[%0], [%1], %2, [%3];" ::"r"(smem_u32(dst_smem)),
      "l"(src_gmem), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
// shared -> global, tracked by the issuing thread's bulk group
__device__ __forceinline__ void bulk_store(void* dst_gmem, const void* src_smem,
                                           uint32_t bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst_gmem),
               "r"(smem_u32(src_smem)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_store_commit_and_wait() {
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
  asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}
// make this thread's generic-proxy shared-memory writes visible to bulk copies
__device__ __forceinline__ void fence_smem_to_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ bool smem_aligned16(const void* p) {
  return (smem_u32(p) & 15u) == 0;
}
__device__ __forceinline__ bool smem_aligned128(const void* p) {
  return (smem_u32(p) & 127u) == 0;
}
// Hint: bring [p, p+bytes) into L2 (p and bytes multiples of 16).
__device__ __forceinline__ void prefetch_l2(const void* p, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_commit() {
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}
// wait until this thread's committed bulk stores have read their shared source
__device__ __forceinline__ void bulk_wait_read_all() {
  asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}

// Tiled rank-4 tensor copies (TMA).  The map is a __grid_constant__ kernel
// parameter; coordinates are element offsets, innermost first.  The caller
// guarantees c0 * element size is a multiple of 16 bytes and, for stores,
// that every coordinate is non-negative.
using TensorMap = CUtensorMap;
#define CLARITY_GRID_CONST const __grid_constant__
__device__ __forceinline__ void tma_load_4d(void* dst, const TensorMap* tm, int c0, int c1,
                                            int c2, int c3, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
      "[%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(tm)), "r"(c0), "r"(c1), "r"(c2), "r"(c3),
      "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void tma_store_4d(const TensorMap* tm, int c0, int c1, int c2,
                                             int c3, const void* src) {
  asm volatile(
      "cp.async.bulk.tensor.4d.global.shared::cta.tile.bulk_group "
      "[%0, {%1, %2, %3, %4}], [%5];" ::"l"(reinterpret_cast<uint64_t>(tm)),
      "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(src))
      : "memory");
}
#else
// Host emulation: copies happen immediately.
inline bool smem_aligned16(const void* p) { return ((uintptr_t)p & 15u) == 0; }
inline bool smem_aligned128(const void* p) { return ((uintptr_t)p & 127u) == 0; }
inline void prefetch_l2(const void*, uint32_t) {}
inline void mbar_init(uint64_t* bar, uint32_t) { *bar = 0; }
inline void mbar_arrive_expect_tx(uint64_t*, uint32_t) {}
inline bool mbar_try_wait(uint64_t*, uint32_t) { return true; }
inline void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t*) {
  std::memcpy(dst, src, bytes);
}
inline void bulk_store(void* dst, const void* src, uint32_t bytes) {
  std::memcpy(dst, src, bytes);
}
inline void bulk_store_commit_and_wait() {}
inline void bulk_commit() {}
inline void bulk_wait_read_all() {}
inline void fence_smem_to_async() {}
// Host emulation of a rank-4 float tensor map and its tiled copies: elements
// outside the tensor read as zero and are not written.
#define CLARITY_GRID_CONST const
struct TensorMap {
  char* base;
  unsigned long long dim[4];
  unsigned long long stride[4];  // bytes; stride[0] = element size
  unsigned box[4];
};
template <bool LOAD>
inline void tma_copy_emu(char* smem, const TensorMap* tm, const int c[4]) {
  size_t o = 0;
  for (unsigned i3 = 0; i3 < tm->box[3]; ++i3)
    for (unsigned i2 = 0; i2 < tm->box[2]; ++i2)
      for (unsigned i1 = 0; i1 < tm->box[1]; ++i1)
        for (unsigned i0 = 0; i0 < tm->box[0]; ++i0, o += 4) {
          const long long g[4] = {(long long)c[0] + i0, (long long)c[1] + i1,
                                  (long long)c[2] + i2, (long long)c[3] + i3};
          bool in = true;
          size_t off = 0;
          for (int d = 0; d < 4; ++d) {
            in = in && g[d] >= 0 && (unsigned long long)g[d] < tm->dim[d];
            off += (size_t)g[d] * tm->stride[d];
          }
          if (LOAD) {
            if (in) std::memcpy(smem + o, tm->base + off, 4);
            else std::memset(smem + o, 0, 4);
          } else if (in) {
            std::memcpy(tm->base + off, smem + o, 4);
          }
        }
}
inline void tma_load_4d(void* dst, const TensorMap* tm, int c0, int c1, int c2, int c3,
                        uint64_t*) {
  const int c[4] = {c0, c1, c2, c3};
  tma_copy_emu<true>(static_cast<char*>(dst), tm, c);
}
inline void tma_store_4d(const TensorMap* tm, int c0, int c1, int c2, int c3, const void* src) {
  const int c[4] = {c0, c1, c2, c3};
  tma_copy_emu<false>(const_cast<char*>(static_cast<const char*>(src)), tm, c);
}
inline int atomicExch(int* p, int v) {
  const int o = *p;
  *p = v;
  return o;
}
#endif

// L2 prefetch of the 16-byte-aligned part of [begin, begin+bytes): never
// touches memory outside the range.
__device__ __forceinline__ void prefetch_l2_range(const void* begin, size_t bytes) {
  const uintptr_t b = reinterpret_cast<uintptr_t>(begin);
  const uintptr_t lo = (b + 15) & ~uintptr_t(15);
  const uintptr_t hi = (b + bytes) & ~uintptr_t(15);
  if (hi > lo) prefetch_l2(reinterpret_cast<const void*>(lo), (uint32_t)(hi - lo));
}

// Encodes a rank-4 float32 tensor map (no interleave, no swizzle, zero fill):
// dim innermost first, stride_bytes for dims 1..3, box extents.  False when
// the driver rejects it (alignment, extents), so callers can fall back.
bool encode_tensor_f32_4d(TensorMap* tm, const void* base, const unsigned long long dim[4],
                          const unsigned long long stride_bytes[3], const unsigned box[4]);
// The same for BF16 elements; swizzle32 selects the 32-byte swizzle (16-byte
// halves of each 32-byte row exchanged when address bit 7 is set), which
// needs a box whose inner extent is 32 bytes and a 256-byte-aligned
// destination.  Device builds only.
bool encode_tensor_bf16_4d(TensorMap* tm, const void* base, const unsigned long long dim[4],
                           const unsigned long long stride_bytes[3], const unsigned box[4],
                           bool swizzle32);

// Records `code` in the context's error word.  The word lives in mapped
// pinned host memory (the host reads it without synchronising the device),
// so it is written with a plain volatile store and a system-scope fence, not
// an atomic: any nonzero code means "this call's result is not valid".
__device__ __forceinline__ void raise_error(int* err, int code) {
  if (!err) return;
  *reinterpret_cast<volatile int*>(err) = code;
#ifndef CLARITY_HOST_EMULATION
  __threadfence_system();
#endif
}

// Bounded wait for phase `parity` of the barrier: at most `limit` polls of
// mbarrier.try_wait; false (and `code` kErrWaitTimeout in *err) when it gives up.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, int* err,
                                                  long long limit) {
  for (long long it = 0; it < limit; ++it)
    if (mbar_try_wait(bar, parity)) return true;
  raise_error(err, kErrWaitTimeout);
  return false;
}

// Bounded wait with the library's limit (kWaitLimit polls).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* err) {
  return mbar_wait_bounded(bar, parity, err, kWaitLimit);
}

}  // namespace clarity
