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
// Hint: bring [p, p+bytes) into L2 (p and bytes multiples of 16).
__device__ __forceinline__ void prefetch_l2(const void* p, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}
#else
// Host emulation: copies happen immediately.
inline bool smem_aligned16(const void* p) { return ((uintptr_t)p & 15u) == 0; }
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
inline void fence_smem_to_async() {}
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

// Bounded wait for phase `parity` of the barrier; false (and *err set) on
// timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* err) {
  for (long long it = 0; it < kWaitLimit; ++it)
    if (mbar_try_wait(bar, parity)) return true;
  if (err) atomicExch(err, kErrWaitTimeout);
  return false;
}

}  // namespace clarity
