// emu_runtime.cpp -- TEST INFRASTRUCTURE: the CUDA runtime calls the library
// makes, implemented on host memory for the CPU emulation build.
#include <chrono>
#include <cstdlib>
#include <cstring>

#include "emu_cuda.hpp"

namespace clarity_emu {
thread_local uint3 tIdx, bIdx;
thread_local dim3 bDim, gDim;
thread_local void* smem_ptr = nullptr;
}  // namespace clarity_emu

extern "C" {
cudaError_t cudaMalloc(void** p, size_t n) {
  *p = std::malloc(n ? n : 16);
  if (*p) std::memset(*p, 0xff, n);  // device memory starts as garbage
  return *p ? cudaSuccess : cudaErrorMemoryAllocation;
}
cudaError_t cudaFree(void* p) {
  std::free(p);
  return cudaSuccess;
}
// mapped pinned host memory: the host pointer is the device alias
cudaError_t cudaHostAlloc(void** p, size_t n, unsigned int) {
  *p = std::malloc(n ? n : 16);
  return *p ? cudaSuccess : cudaErrorMemoryAllocation;
}
cudaError_t cudaFreeHost(void* p) {
  std::free(p);
  return cudaSuccess;
}
cudaError_t cudaHostGetDevicePointer(void** d, void* h, unsigned int) {
  *d = h;
  return cudaSuccess;
}
// every host pointer is ordinary (pageable) memory in the emulation, so
// the host API's pinned bounce path runs
cudaError_t cudaPointerGetAttributes(cudaPointerAttributes* a, const void*) {
  std::memset(a, 0, sizeof(*a));
  a->type = cudaMemoryTypeUnregistered;
  return cudaSuccess;
}
cudaError_t cudaStreamIsCapturing(cudaStream_t, cudaStreamCaptureStatus* s) {
  *s = cudaStreamCaptureStatusNone;
  return cudaSuccess;
}
cudaError_t cudaMemcpyAsync(void* d, const void* s, size_t n, cudaMemcpyKind, cudaStream_t) {
  std::memcpy(d, s, n);
  return cudaSuccess;
}
cudaError_t cudaStreamCreateWithFlags(cudaStream_t* s, unsigned int) {
  *s = reinterpret_cast<cudaStream_t>(new int(1));
  return cudaSuccess;
}
cudaError_t cudaStreamDestroy(cudaStream_t s) {
  delete reinterpret_cast<int*>(s);
  return cudaSuccess;
}
cudaError_t cudaStreamSynchronize(cudaStream_t) { return cudaSuccess; }
cudaError_t cudaMemsetAsync(void* p, int v, size_t n, cudaStream_t) {
  std::memset(p, v, n);
  return cudaSuccess;
}
cudaError_t cudaMemset(void* p, int v, size_t n) {
  std::memset(p, v, n);
  return cudaSuccess;
}
cudaError_t cudaMemcpy(void* d, const void* s, size_t n, cudaMemcpyKind) {
  std::memcpy(d, s, n);
  return cudaSuccess;
}
cudaError_t cudaDeviceSynchronize(void) { return cudaSuccess; }
cudaError_t cudaSetDevice(int) { return cudaSuccess; }
cudaError_t cudaGetDeviceCount(int* c) {
  *c = 1;
  return cudaSuccess;
}
cudaError_t cudaGetDeviceProperties_v2(cudaDeviceProp* p, int) {
  std::memset(p, 0, sizeof(*p));
  std::strcpy(p->name, "host emulation");
  p->major = 10;
  p->minor = 0;
  p->totalGlobalMem = 1ull << 34;
  return cudaSuccess;
}
cudaError_t cudaGetLastError(void) { return cudaSuccess; }
cudaError_t cudaGetDevice(int* d) {
  *d = 0;
  return cudaSuccess;
}
cudaError_t cudaGetSymbolAddress(void** p, const void* symbol) {
  *p = const_cast<void*>(symbol);
  return cudaSuccess;
}
const char* cudaGetErrorString(cudaError_t e) {
  return e == cudaSuccess ? "no error" : "emulated error";
}
cudaError_t cudaFuncSetAttribute(const void*, cudaFuncAttribute, int) { return cudaSuccess; }
cudaError_t cudaEventCreate(cudaEvent_t* e) {
  *e = reinterpret_cast<cudaEvent_t>(new double(0));
  return cudaSuccess;
}
cudaError_t cudaEventRecord(cudaEvent_t e, cudaStream_t) {
  *reinterpret_cast<double*>(e) =
      std::chrono::duration<double, std::milli>(
          std::chrono::steady_clock::now().time_since_epoch()).count();
  return cudaSuccess;
}
cudaError_t cudaEventSynchronize(cudaEvent_t) { return cudaSuccess; }
cudaError_t cudaEventCreateWithFlags(cudaEvent_t* e, unsigned int) { return cudaEventCreate(e); }
cudaError_t cudaEventDestroy(cudaEvent_t e) {
  delete reinterpret_cast<double*>(e);
  return cudaSuccess;
}
// the emulation never instantiates graphs (batches run as issued)
cudaError_t cudaGraphExecDestroy(cudaGraphExec_t) { return cudaSuccess; }
// every emulated kernel has finished when its launch returns: waits are no-ops
cudaError_t cudaStreamWaitEvent(cudaStream_t, cudaEvent_t, unsigned int) { return cudaSuccess; }
cudaError_t cudaEventElapsedTime(float* ms, cudaEvent_t a, cudaEvent_t b) {
  *ms = (float)(*reinterpret_cast<double*>(b) - *reinterpret_cast<double*>(a));
  return cudaSuccess;
}
}
