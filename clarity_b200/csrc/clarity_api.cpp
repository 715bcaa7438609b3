// clarity_api.cpp -- the C ABI of libclarity.so (include/clarity.h and
// include/clarity_ext.h).
//
// Public functions follow the reference contract (Clarity.h.in:123-383):
// host buffers in and out, synchronous, ClarityResult_t codes with
// CLARITY_SUCCESS == 5.  Inside, unpadded volumes are copied to the device
// once and padded on the fly by the first FFT pass (the reference pads on
// the host, src/ImagePadSpatialShift.cxx, and copies three padded volumes).
#include <cuda_runtime.h>

#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <mutex>
#include <vector>
#include <string>

#include "../../include/clarity.h"
#include "../../include/clarity_ext.h"
#include "engine.hpp"

using clarity::Context;
using clarity::Dims;
using clarity::Status;

namespace {

std::mutex g_mu;                 // guards registration state
int g_refcount = 0;              // src/Clarity.cxx:41 (made thread-safe)
int g_device = 0;
Context* g_ctx = nullptr;
bool g_autotune = false;         // applied to contexts created later too
unsigned g_threads = 0;
thread_local char g_last_error[512];

// Staging buffers for the host-buffer API (grown on demand).
struct Staging {
  float* img = nullptr;
  float* ker = nullptr;
  float* out = nullptr;
  size_t img_cap = 0, ker_cap = 0, out_cap = 0;
} g_stage;

// Library-owned pinned bounce buffers for callers whose host buffers are
// pageable (every reference caller allocates with malloc or new,
// src/Memory.cxx:97-156 copies from them synchronously).  A copy is cut
// into chunks that alternate between two pinned buffers: the host copies
// chunk k into one while the DMA engine moves chunk k-1 out of the other.
// Buffers the caller pinned itself (cudaHostAlloc, cudaHostRegister) are
// copied directly.
struct PinnedBounce {
  static constexpr size_t kChunk = size_t(8) << 20;
  void* buf[2] = {nullptr, nullptr};
  cudaEvent_t ev[2] = {nullptr, nullptr};
} g_bounce;

bool host_is_pinned(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();  // an unregistered pointer is not an error here
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

cudaError_t bounce_ready() {
  for (int i = 0; i < 2; ++i) {
    if (!g_bounce.buf[i]) {
      cudaError_t e = cudaHostAlloc(&g_bounce.buf[i], PinnedBounce::kChunk, cudaHostAllocPortable);
      if (e != cudaSuccess) return e;
    }
    if (!g_bounce.ev[i]) {
      cudaError_t e = cudaEventCreateWithFlags(&g_bounce.ev[i], cudaEventDisableTiming);
      if (e != cudaSuccess) return e;
    }
  }
  return cudaSuccess;
}

void free_bounce() {
  for (int i = 0; i < 2; ++i) {
    if (g_bounce.buf[i]) cudaFreeHost(g_bounce.buf[i]);
    if (g_bounce.ev[i]) cudaEventDestroy(g_bounce.ev[i]);
  }
  g_bounce = PinnedBounce();
}

// host -> device on `st`, asynchronous for pinned sources; a pageable source
// has been read completely when this returns.
cudaError_t upload(void* dst, const void* src, size_t bytes, cudaStream_t st) {
  if (bytes == 0) return cudaSuccess;
  if (host_is_pinned(src)) return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st);
  cudaError_t e = bounce_ready();
  if (e != cudaSuccess) return e;
  const char* s = static_cast<const char*>(src);
  char* d = static_cast<char*>(dst);
  for (size_t off = 0, k = 0; off < bytes; off += PinnedBounce::kChunk, ++k) {
    const int i = (int)(k & 1);
    const size_t n = std::min(PinnedBounce::kChunk, bytes - off);
    if ((e = cudaEventSynchronize(g_bounce.ev[i])) != cudaSuccess) return e;  // buffer free
    std::memcpy(g_bounce.buf[i], s + off, n);
    if ((e = cudaMemcpyAsync(d + off, g_bounce.buf[i], n, cudaMemcpyHostToDevice, st)) !=
        cudaSuccess)
      return e;
    if ((e = cudaEventRecord(g_bounce.ev[i], st)) != cudaSuccess) return e;
  }
  return cudaSuccess;
}

// device -> host on `st`; complete (the host buffer written) when it returns
// for a pageable destination, asynchronous for a pinned one.
cudaError_t download(void* dst, const void* src, size_t bytes, cudaStream_t st) {
  if (bytes == 0) return cudaSuccess;
  if (host_is_pinned(dst)) return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st);
  cudaError_t e = bounce_ready();
  if (e != cudaSuccess) return e;
  const char* s = static_cast<const char*>(src);
  char* d = static_cast<char*>(dst);
  const size_t nch = (bytes + PinnedBounce::kChunk - 1) / PinnedBounce::kChunk;
  auto issue = [&](size_t k) -> cudaError_t {
    const int i = (int)(k & 1);
    const size_t off = k * PinnedBounce::kChunk, n = std::min(PinnedBounce::kChunk, bytes - off);
    cudaError_t r = cudaEventSynchronize(g_bounce.ev[i]);
    if (r == cudaSuccess) r = cudaMemcpyAsync(g_bounce.buf[i], s + off, n,
                                              cudaMemcpyDeviceToHost, st);
    if (r == cudaSuccess) r = cudaEventRecord(g_bounce.ev[i], st);
    return r;
  };
  if ((e = issue(0)) != cudaSuccess) return e;
  for (size_t k = 0; k < nch; ++k) {
    if (k + 1 < nch && (e = issue(k + 1)) != cudaSuccess) return e;
    const int i = (int)(k & 1);
    const size_t off = k * PinnedBounce::kChunk, n = std::min(PinnedBounce::kChunk, bytes - off);
    if ((e = cudaEventSynchronize(g_bounce.ev[i])) != cudaSuccess) return e;
    std::memcpy(d + off, g_bounce.buf[i], n);
  }
  return cudaSuccess;
}

bool g_implicit = false;         // the context was created by a call, not by Register

void set_error(const char* msg) {
  std::snprintf(g_last_error, sizeof(g_last_error), "%s", msg ? msg : "");
}

ClarityResult_t fail(ClarityResult_t code, const std::string& msg) {
  set_error(msg.c_str());
  return code;
}

ClarityResult_t report(const Status& s) {
  if (s.ok()) return CLARITY_SUCCESS;
  set_error(s.msg.c_str());
  return s.code;
}

bool dims_ok(Clarity_Dim3 d) { return d.x > 0 && d.y > 0 && d.z > 0; }

long long nvox(Clarity_Dim3 d) { return (long long)d.x * d.y * d.z; }

Dims to_dims(Clarity_Dim3 d) { return Dims{d.x, d.y, d.z}; }

Status grow(float** p, size_t* cap, size_t n) {
  if (*cap >= n && *p) return Status::Ok();
  cudaFree(*p);
  *p = nullptr;
  *cap = 0;
  cudaError_t e = clarity::dev_alloc((void**)p, sizeof(float) * n);
  if (e != cudaSuccess) return clarity::status_from_cuda(e, "staging allocation");
  *cap = n;
  return Status::Ok();
}

void free_staging() {
  cudaFree(g_stage.img);
  cudaFree(g_stage.ker);
  cudaFree(g_stage.out);
  g_stage = Staging();
  free_bounce();
}

// Creates the library context on the selected device (g_mu held).
ClarityResult_t create_context_locked(const char* who) {
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count <= g_device)
    return fail(CLARITY_INVALID_OPERATION, std::string(who) + ": no CUDA device available");
  cudaDeviceProp prop;
  e = cudaGetDeviceProperties(&prop, g_device);
  if (e != cudaSuccess)
    return fail(CLARITY_INVALID_OPERATION, std::string(who) + ": " + cudaGetErrorString(e));
  if (prop.major != 10)
    return fail(CLARITY_INVALID_OPERATION,
                std::string(who) + ": device is not sm_100 class: " + prop.name);
  Context* c = new Context(g_device);
  const Status is = c->init();
  if (!is.ok()) {
    delete c;
    return report(is);
  }
  c->set_autotune(g_autotune);
  g_ctx = c;
  if (std::getenv("CLARITY_LOG"))
    std::fprintf(stderr, "clarity: device %d '%s', %zu MB\n", g_device, prop.name,
                 (size_t)(prop.totalGlobalMem >> 20));
  return CLARITY_SUCCESS;
}

// The context a call runs on.  Callers of the reference need not call
// Clarity_Register first -- its functions work without it, and its own
// raw-image app (apps/DeconvolveRawImages/DeconvolveRawImages.cxx) never
// calls it -- so the first call without a registration creates the context
// itself.  A later Clarity_Register adopts it; Clarity_UnRegister releases it
// when the registrations balance, and otherwise it lives until the process
// exits.
Context* acquire_context(ClarityResult_t* rc) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_ctx) {
    *rc = create_context_locked("Clarity_Register (implicit, on first use)");
    if (*rc != CLARITY_SUCCESS) return nullptr;
    g_implicit = true;
  }
  return g_ctx;
}

// Common path of the host-buffer algorithms: validate, upload, run, download.
template <class Run>
ClarityResult_t host_call(const float* in, Clarity_Dim3 id, const float* ker,
                          Clarity_Dim3 kd, float* out, Run run) {
  if (!in || !ker || !out) return fail(CLARITY_INVALID_ARGUMENT, "NULL buffer");
  if (!dims_ok(id) || !dims_ok(kd))
    return fail(CLARITY_INVALID_ARGUMENT, "dimension <= 0");
  ClarityResult_t rc_ = CLARITY_SUCCESS;
  Context* ctx = acquire_context(&rc_);
  if (!ctx) return rc_;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device());
  ctx->clear_stream();
  // a failure recorded by earlier asynchronous work is reported, not hidden
  // behind this call's success
  Status s = ctx->check_device_errors();
  if (!s.ok()) return report(s);
  const size_t ni = (size_t)nvox(id), nk = (size_t)nvox(kd);
  s = grow(&g_stage.img, &g_stage.img_cap, ni);
  if (s.ok()) s = grow(&g_stage.ker, &g_stage.ker_cap, nk);
  if (s.ok()) s = grow(&g_stage.out, &g_stage.out_cap, ni);
  if (!s.ok()) return report(s);
  cudaStream_t st = ctx->exec_stream();
  cudaError_t e = upload(g_stage.img, in, sizeof(float) * ni, st);
  if (e == cudaSuccess) e = upload(g_stage.ker, ker, sizeof(float) * nk, st);
  if (e != cudaSuccess) return report(clarity::status_from_cuda(e, "host to device copy"));
  s = run(*ctx, g_stage.img, to_dims(id), g_stage.ker, to_dims(kd), g_stage.out);
  if (!s.ok()) return report(s);
  e = download(out, g_stage.out, sizeof(float) * ni, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return report(clarity::status_from_cuda(e, "device to host copy"));
  return report(ctx->check_device_errors());
}

template <class Run>
ClarityResult_t device_call(const float* in, Clarity_Dim3 id, const float* ker,
                            Clarity_Dim3 kd, float* out, void* stream, Run run) {
  if (!in || !ker || !out) return fail(CLARITY_INVALID_ARGUMENT, "NULL buffer");
  if (!dims_ok(id) || !dims_ok(kd))
    return fail(CLARITY_INVALID_ARGUMENT, "dimension <= 0");
  ClarityResult_t rc_ = CLARITY_SUCCESS;
  Context* ctx = acquire_context(&rc_);
  if (!ctx) return rc_;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device());
  // a bounded wait of earlier work that gave up is reported here (that
  // work's result is not valid) and nothing is enqueued
  Status s = ctx->check_device_errors();
  if (!s.ok()) return report(s);
  ctx->set_stream(static_cast<cudaStream_t>(stream));
  s = run(*ctx, in, to_dims(id), ker, to_dims(kd), out);
  ctx->clear_stream();
  return report(s);
}

}  // namespace

namespace clarity {
Context* global_context() { return g_ctx; }
// Records the message returned by clarityx_last_error (fixed buffer, no
// allocation).
void set_last_error(const char* msg) { set_error(msg); }
}  // namespace clarity

// ================================================================== public

extern "C" {

Clarity_Dim3 Clarity_Dim3FromArray(int dimArray[3]) {
  Clarity_Dim3 d;
  d.x = dimArray[0];
  d.y = dimArray[1];
  d.z = dimArray[2];
  return d;
}

ClarityResult_t Clarity_Register(void) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (g_refcount == 0) {
    if (g_ctx) {
      g_implicit = false;  // adopt the context an earlier call created
    } else {
      const ClarityResult_t r = create_context_locked("Clarity_Register");
      if (r != CLARITY_SUCCESS) return r;
    }
  }
  g_refcount++;
  return CLARITY_SUCCESS;
}

ClarityResult_t Clarity_UnRegister(void) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (g_refcount <= 0) return fail(CLARITY_INVALID_OPERATION, "not registered");
  if (--g_refcount == 0) {
    {
      std::lock_guard<std::mutex> lk2(g_ctx->mu);
      cudaSetDevice(g_ctx->device());
      cudaDeviceSynchronize();
      free_staging();
    }
    delete g_ctx;
    g_ctx = nullptr;
  }
  return CLARITY_SUCCESS;
}

ClarityResult_t Clarity_SetNumberOfThreads(unsigned n) {
  g_threads = n;
  return CLARITY_SUCCESS;
}

ClarityResult_t Clarity_ImagePadSpatialShift(float* dst, Clarity_Dim3 dstDim,
                                             float* src, Clarity_Dim3 srcDim,
                                             int shift[3], float fillValue) {
  if (!dst || !src || !shift) return fail(CLARITY_INVALID_ARGUMENT, "NULL buffer");
  if (!dims_ok(dstDim) || !dims_ok(srcDim))
    return fail(CLARITY_INVALID_ARGUMENT, "dimension <= 0");
  // src/ImagePadSpatialShift.cxx:42-66
  for (int dk = 0; dk < dstDim.z; dk++) {
    int sk = dk - shift[2];
    if (sk < 0) sk += dstDim.z;
    sk = sk % dstDim.z;
    const bool wk = sk >= 0 && sk < srcDim.z;
    for (int dj = 0; dj < dstDim.y; dj++) {
      int sj = dj - shift[1];
      if (sj < 0) sj += dstDim.y;
      sj = sj % dstDim.y;
      const bool wj = sj >= 0 && sj < srcDim.y;
      float* drow = dst + ((long long)dk * dstDim.y + dj) * dstDim.x;
      const float* srow = src + ((long long)sk * srcDim.y + sj) * srcDim.x;
      for (int di = 0; di < dstDim.x; di++) {
        int si = di - shift[0];
        if (si < 0) si += dstDim.x;
        si = si % dstDim.x;
        const bool wi = si >= 0 && si < srcDim.x;
        drow[di] = (wi && wj && wk) ? srow[si] : fillValue;
      }
    }
  }
  return CLARITY_SUCCESS;
}

ClarityResult_t Clarity_ImageClip(float* dst, Clarity_Dim3 dstDim, float* src,
                                  Clarity_Dim3 srcDim) {
  if (!dst || !src) return fail(CLARITY_INVALID_ARGUMENT, "NULL buffer");
  if (!dims_ok(dstDim) || !dims_ok(srcDim))
    return fail(CLARITY_INVALID_ARGUMENT, "dimension <= 0");
  if (dstDim.x > srcDim.x || dstDim.y > srcDim.y || dstDim.z > srcDim.z)
    return fail(CLARITY_INVALID_ARGUMENT, "clip box larger than source");
  for (int k = 0; k < dstDim.z; k++)
    for (int j = 0; j < dstDim.y; j++)
      std::memcpy(dst + ((long long)k * dstDim.y + j) * dstDim.x,
                  src + ((long long)k * srcDim.y + j) * srcDim.x,
                  sizeof(float) * dstDim.x);
  return CLARITY_SUCCESS;
}

char* Clarity_ResultString(ClarityResult_t result) {
  // src/Clarity.cxx:116-150
  switch (result) {
    case CLARITY_FFT_FAILED: return const_cast<char*>("CLARITY_FFT_FAILED");
    case CLARITY_OUT_OF_MEMORY: return const_cast<char*>("CLARITY_OUT_OF_MEMORY");
    case CLARITY_DEVICE_OUT_OF_MEMORY:
      return const_cast<char*>("CLARITY_DEVICE_OUT_OF_MEMORY");
    case CLARITY_INVALID_OPERATION: return const_cast<char*>("CLARITY_INVALID_OPERATION");
    case CLARITY_INVALID_ARGUMENT: return const_cast<char*>("CLARITY_INVALID_ARGUMENT");
    case CLARITY_SUCCESS: return const_cast<char*>("CLARITY_SUCCESS");
    default: return const_cast<char*>("<unknown Clarity result>");
  }
}

ClarityResult_t Clarity_WienerDeconvolve(float* inImage, Clarity_Dim3 imageDim,
                                         float* kernelImage, Clarity_Dim3 kernelDim,
                                         float* outImage, float epsilon) {
  return host_call(inImage, imageDim, kernelImage, kernelDim, outImage,
                   [&](Context& c, const float* i, Dims id, const float* k, Dims kd,
                       float* o) { return clarity::run_wiener(c, i, id, k, kd, o, epsilon); });
}

ClarityResult_t Clarity_JansenVanCittertDeconvolve(float* inImage, Clarity_Dim3 imageDim,
                                                   float* kernelImage,
                                                   Clarity_Dim3 kernelDim,
                                                   float* outImage, int iterations) {
  return host_call(inImage, imageDim, kernelImage, kernelDim, outImage,
                   [&](Context& c, const float* i, Dims id, const float* k, Dims kd,
                       float* o) {
                     return clarity::run_jvc(c, i, id, k, kd, o, iterations, 0.f,
                                             nullptr, 0);
                   });
}

ClarityResult_t Clarity_SmoothedJansenVanCittertDeconvolve(
    float* inImage, Clarity_Dim3 imageDim, float* kernelImage, Clarity_Dim3 kernelDim,
    float* outImage, unsigned iterations, unsigned smoothInterval,
    float* smoothSigma[3]) {
  float sig[3] = {0.f, 0.f, 0.f};
  bool smooth = smoothSigma != nullptr && smoothInterval > 0;
  if (smooth) {
    for (int d = 0; d < 3; ++d) {
      if (!smoothSigma[d]) { smooth = false; break; }
      sig[d] = *smoothSigma[d];
    }
  }
  return host_call(inImage, imageDim, kernelImage, kernelDim, outImage,
                   [&](Context& c, const float* i, Dims id, const float* k, Dims kd,
                       float* o) {
                     return clarity::run_jvc(c, i, id, k, kd, o, (int)iterations, 0.f,
                                             smooth ? sig : nullptr,
                                             smooth ? (int)smoothInterval : 0);
                   });
}

ClarityResult_t Clarity_IDivergenceDeconvolve(float* inImage, Clarity_Dim3 imageDim,
                                              float* kernelImage, Clarity_Dim3 kernelDim,
                                              float* outImage) {
  // The reference body writes zeros (src/IDivergenceDeconvolve.cxx:59-72).
  if (!inImage || !kernelImage || !outImage)
    return fail(CLARITY_INVALID_ARGUMENT, "NULL buffer");
  if (!dims_ok(imageDim) || !dims_ok(kernelDim))
    return fail(CLARITY_INVALID_ARGUMENT, "dimension <= 0");
  std::memset(outImage, 0, sizeof(float) * (size_t)nvox(imageDim));
  return CLARITY_SUCCESS;
}

ClarityResult_t Clarity_MaximumLikelihoodDeconvolve(float* inImage, Clarity_Dim3 imageDim,
                                                    float* kernelImage,
                                                    Clarity_Dim3 kernelDim,
                                                    float* outImage, int iterations) {
  return host_call(inImage, imageDim, kernelImage, kernelDim, outImage,
                   [&](Context& c, const float* i, Dims id, const float* k, Dims kd,
                       float* o) { return clarity::run_rl(c, i, id, k, kd, o, iterations); });
}

ClarityResult_t Clarity_BlindMaximumLikelihoodDeconvolve(float* inImage,
                                                         Clarity_Dim3 imageDim,
                                                         float* kernelImage,
                                                         Clarity_Dim3 kernelDim,
                                                         float* outImage, int iterations) {
  return host_call(inImage, imageDim, kernelImage, kernelDim, outImage,
                   [&](Context& c, const float* i, Dims id, const float* k, Dims kd,
                       float* o) {
                     return clarity::run_blind(c, i, id, k, kd, o, iterations);
                   });
}

ClarityResult_t Clarity_Convolve(float* inImage, Clarity_Dim3 imageDim, float* kernel,
                                 Clarity_Dim3 kernelDim, float* outImage) {
  return host_call(inImage, imageDim, kernel, kernelDim, outImage,
                   [&](Context& c, const float* i, Dims id, const float* k, Dims kd,
                       float* o) { return clarity::run_convolve(c, i, id, k, kd, o); });
}

// ============================================================== extensions

const char* clarityx_last_error(void) { return g_last_error; }

ClarityResult_t clarityx_set_device(int device) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (g_refcount > 0 || g_ctx)
    return fail(CLARITY_INVALID_OPERATION, "already registered (or a call created the context)");
  if (device < 0) return fail(CLARITY_INVALID_ARGUMENT, "negative device");
  g_device = device;
  return CLARITY_SUCCESS;
}

void clarityx_inject_device_alloc_failure(int countdown) {
  clarity::set_alloc_failure_countdown(countdown);
}

ClarityResult_t clarityx_trim(void) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_ctx) return fail(CLARITY_INVALID_OPERATION, "not registered");
  std::lock_guard<std::mutex> lk2(g_ctx->mu);
  cudaSetDevice(g_ctx->device());
  cudaDeviceSynchronize();
  g_ctx->release_workspaces();
  free_staging();
  return CLARITY_SUCCESS;
}

ClarityResult_t clarityx_synchronize(void* stream) {
  Context* ctx;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    ctx = g_ctx;
  }
  if (!ctx) return fail(CLARITY_INVALID_OPERATION, "not registered");
  cudaSetDevice(ctx->device());
  // NULL: every stream of the device (the library's own included)
  const cudaError_t e = stream ? cudaStreamSynchronize(static_cast<cudaStream_t>(stream))
                               : cudaDeviceSynchronize();
  if (e != cudaSuccess) return report(clarity::status_from_cuda(e, "synchronize"));
  return report(ctx->check_device_errors());
}

ClarityResult_t clarityx_inject_wait_timeout(void* stream) {
  Context* ctx;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    ctx = g_ctx;
  }
  if (!ctx) return fail(CLARITY_INVALID_OPERATION, "not registered");
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device());
  ctx->set_stream(static_cast<cudaStream_t>(stream));
  const Status s = clarity::inject_wait_timeout(*ctx);
  ctx->clear_stream();
  return report(s);
}

ClarityResult_t clarityx_convolve_device(const float* image, Clarity_Dim3 imageDim,
                                         const float* kernel, Clarity_Dim3 kernelDim,
                                         float* out, void* stream) {
  return device_call(image, imageDim, kernel, kernelDim, out, stream,
                     [&](Context& c, const float* i, Dims id, const float* k, Dims kd,
                         float* o) { return clarity::run_convolve(c, i, id, k, kd, o); });
}

ClarityResult_t clarityx_wiener_device(const float* image, Clarity_Dim3 imageDim,
                                       const float* kernel, Clarity_Dim3 kernelDim,
                                       float* out, float epsilon, void* stream) {
  return device_call(image, imageDim, kernel, kernelDim, out, stream,
                     [&](Context& c, const float* i, Dims id, const float* k, Dims kd,
                         float* o) {
                       return clarity::run_wiener(c, i, id, k, kd, o, epsilon);
                     });
}

ClarityResult_t clarityx_ml_device(const float* image, Clarity_Dim3 imageDim,
                                   const float* kernel, Clarity_Dim3 kernelDim,
                                   float* out, int iterations, void* stream) {
  return device_call(image, imageDim, kernel, kernelDim, out, stream,
                     [&](Context& c, const float* i, Dims id, const float* k, Dims kd,
                         float* o) {
                       return clarity::run_rl(c, i, id, k, kd, o, iterations);
                     });
}

ClarityResult_t clarityx_correlate_device(const float* image, Clarity_Dim3 imageDim,
                                          const float* kernel, Clarity_Dim3 kernelDim,
                                          float* out, void* stream) {
  return device_call(image, imageDim, kernel, kernelDim, out, stream,
                     [&](Context& c, const float* i, Dims id, const float* k, Dims kd,
                         float* o) { return clarity::run_correlate(c, i, id, k, kd, o); });
}

ClarityResult_t clarityx_ml_correlate_device(const float* image, Clarity_Dim3 imageDim,
                                             const float* kernel, Clarity_Dim3 kernelDim,
                                             float* out, int iterations, void* stream) {
  return device_call(image, imageDim, kernel, kernelDim, out, stream,
                     [&](Context& c, const float* i, Dims id, const float* k, Dims kd,
                         float* o) {
                       return clarity::run_rl_correlate(c, i, id, k, kd, o, iterations);
                     });
}

ClarityResult_t clarityx_ml_learned_device(const float* image, Clarity_Dim3 imageDim,
                                           const float* kernel, Clarity_Dim3 kernelDim,
                                           const float* params, long long nparams, int pre,
                                           float* out, int post, double* idiv, void* stream) {
  if (!params) return fail(CLARITY_INVALID_ARGUMENT, "NULL network parameters");
  if (nparams != clarity::nn_param_count())
    return fail(CLARITY_INVALID_ARGUMENT,
                "network parameters: expected " + std::to_string(clarity::nn_param_count()) +
                    " floats, got " + std::to_string(nparams));
  return device_call(image, imageDim, kernel, kernelDim, out, stream,
                     [&](Context& c, const float* i, Dims id, const float* k, Dims kd,
                         float* o) {
                       return clarity::run_ml_learned(c, i, id, k, kd, params, pre, o, post,
                                                      idiv);
                     });
}

long long clarityx_nn_param_count(void) { return clarity::nn_param_count(); }

ClarityResult_t clarityx_nn_predict(const float* params, long long nparams, const float* x,
                                    Clarity_Dim3 dim, float* out, void* stream) {
  if (!params || !x || !out) return fail(CLARITY_INVALID_ARGUMENT, "NULL buffer");
  if (!dims_ok(dim)) return fail(CLARITY_INVALID_ARGUMENT, "dimension <= 0");
  if (nparams != clarity::nn_param_count())
    return fail(CLARITY_INVALID_ARGUMENT, "network parameters: wrong count");
  ClarityResult_t rc_ = CLARITY_SUCCESS;
  Context* ctx = acquire_context(&rc_);
  if (!ctx) return rc_;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device());
  Status s = ctx->check_device_errors();
  if (!s.ok()) return report(s);
  ctx->set_stream(static_cast<cudaStream_t>(stream));
  s = clarity::nn_predict(*ctx, params, x, dim.z, dim.y, dim.x, out);
  ctx->clear_stream();
  return report(s);
}

ClarityResult_t clarityx_idiv_deconvolve_device(const float* image, Clarity_Dim3 imageDim,
                                               const float* kernel, Clarity_Dim3 kernelDim,
                                               float* out, int iterations, float alpha,
                                               void* stream) {
  if (iterations < 0) return fail(CLARITY_INVALID_ARGUMENT, "iterations < 0");
  if (!(alpha >= 0.f)) return fail(CLARITY_INVALID_ARGUMENT, "alpha < 0 or NaN");
  return device_call(image, imageDim, kernel, kernelDim, out, stream,
                     [&](Context& c, const float* i, Dims id, const float* k, Dims kd,
                         float* o) {
                       return clarity::run_idiv_cg(c, i, id, k, kd, o, iterations, alpha);
                     });
}

ClarityResult_t clarityx_blind_ml_psf_device(const float* image, Clarity_Dim3 imageDim,
                                             const float* kernel, Clarity_Dim3 kernelDim,
                                             float* out, float* psf_out, int iterations,
                                             int psf_subiterations, void* stream) {
  if (psf_subiterations < 0) return fail(CLARITY_INVALID_ARGUMENT, "psf_subiterations < 0");
  return device_call(image, imageDim, kernel, kernelDim, out, stream,
                     [&](Context& c, const float* i, Dims id, const float* k, Dims kd,
                         float* o) {
                       return clarity::run_blind_psf(c, i, id, k, kd, o, psf_out, iterations,
                                                     psf_subiterations);
                     });
}

ClarityResult_t clarityx_ml_u16(const uint16_t* image, Clarity_Dim3 imageDim,
                                const uint16_t* kernel, Clarity_Dim3 kernelDim, uint16_t* out,
                                int iterations) {
  if (!image || !kernel || !out) return fail(CLARITY_INVALID_ARGUMENT, "NULL buffer");
  if (!dims_ok(imageDim) || !dims_ok(kernelDim))
    return fail(CLARITY_INVALID_ARGUMENT, "dimension <= 0");
  ClarityResult_t rc_ = CLARITY_SUCCESS;
  Context* ctx = acquire_context(&rc_);
  if (!ctx) return rc_;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device());
  ctx->clear_stream();
  Status s = ctx->check_device_errors();
  if (!s.ok()) return report(s);
  const size_t ni = (size_t)nvox(imageDim), nk = (size_t)nvox(kernelDim);
  // uint16 data lands in the output staging buffer (sized for either
  // volume), is cast into the image / kernel staging buffers, and the result
  // is cast back into the image staging buffer
  s = grow(&g_stage.img, &g_stage.img_cap, ni);
  if (s.ok()) s = grow(&g_stage.ker, &g_stage.ker_cap, nk);
  if (s.ok()) s = grow(&g_stage.out, &g_stage.out_cap, std::max(ni, nk));
  if (!s.ok()) return report(s);
  cudaStream_t st = ctx->exec_stream();
  uint16_t* raw = reinterpret_cast<uint16_t*>(g_stage.out);
  cudaError_t e = upload(raw, image, sizeof(uint16_t) * ni, st);
  if (e != cudaSuccess) return report(clarity::status_from_cuda(e, "host to device copy"));
  s = clarity::cast_u16_to_f32(*ctx, raw, g_stage.img, (long long)ni);
  if (!s.ok()) return report(s);
  e = upload(raw, kernel, sizeof(uint16_t) * nk, st);
  if (e != cudaSuccess) return report(clarity::status_from_cuda(e, "host to device copy"));
  s = clarity::cast_u16_to_f32(*ctx, raw, g_stage.ker, (long long)nk);
  if (s.ok())
    s = clarity::run_rl(*ctx, g_stage.img, to_dims(imageDim), g_stage.ker, to_dims(kernelDim),
                        g_stage.out, iterations);
  if (!s.ok()) return report(s);
  uint16_t* res = reinterpret_cast<uint16_t*>(g_stage.img);
  s = clarity::cast_f32_to_u16(*ctx, g_stage.out, res, (long long)ni);
  if (!s.ok()) return report(s);
  e = download(out, res, sizeof(uint16_t) * ni, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return report(clarity::status_from_cuda(e, "device to host copy"));
  return report(ctx->check_device_errors());
}

ClarityResult_t clarityx_ml_ex_device(const float* image, Clarity_Dim3 imageDim,
                                      const float* kernel, Clarity_Dim3 kernelDim,
                                      const float* start, float* out, int iterations,
                                      double* idiv, void* stream) {
  return device_call(image, imageDim, kernel, kernelDim, out, stream,
                     [&](Context& c, const float* i, Dims id, const float* k, Dims kd,
                         float* o) {
                       return clarity::run_rl_ex(c, i, id, k, kd, start, o, iterations, idiv);
                     });
}

ClarityResult_t clarityx_ml_accel_device(const float* image, Clarity_Dim3 imageDim,
                                         const float* kernel, Clarity_Dim3 kernelDim,
                                         const float* start, float* out, int iterations,
                                         double* idiv, void* stream) {
  return device_call(image, imageDim, kernel, kernelDim, out, stream,
                     [&](Context& c, const float* i, Dims id, const float* k, Dims kd,
                         float* o) {
                       return clarity::run_rl_accel(c, i, id, k, kd, start, o, iterations, idiv);
                     });
}

ClarityResult_t clarityx_ml_batch_device(int count, const float* const* images,
                                         const Clarity_Dim3* imageDims,
                                         const float* const* kernels,
                                         const Clarity_Dim3* kernelDims, float* const* outs,
                                         int iterations, int flags, void* stream) {
  if (count < 0) return fail(CLARITY_INVALID_ARGUMENT, "count < 0");
  if (count == 0) return CLARITY_SUCCESS;
  if (!images || !imageDims || !kernels || !kernelDims || !outs)
    return fail(CLARITY_INVALID_ARGUMENT, "NULL array");
  std::vector<Dims> ids(count), kds(count);
  for (int i = 0; i < count; ++i) {
    if (!dims_ok(imageDims[i]) || !dims_ok(kernelDims[i]))
      return fail(CLARITY_INVALID_ARGUMENT, "dimension <= 0");
    ids[i] = to_dims(imageDims[i]);
    kds[i] = to_dims(kernelDims[i]);
  }
  ClarityResult_t rc_ = CLARITY_SUCCESS;
  Context* ctx = acquire_context(&rc_);
  if (!ctx) return rc_;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device());
  Status s = ctx->check_device_errors();
  if (!s.ok()) return report(s);
  ctx->set_stream(static_cast<cudaStream_t>(stream));
  s = clarity::run_rl_batch(*ctx, count, images, ids.data(), kernels, kds.data(), outs,
                            iterations, (flags & CLARITYX_BATCH_GRAPH) != 0,
                            (flags & CLARITYX_BATCH_PERSISTENT) != 0);
  ctx->clear_stream();
  return report(s);
}

ClarityResult_t clarityx_set_dft_precision(int mode) {
  if (mode < 0 || mode > 2) return fail(CLARITY_INVALID_ARGUMENT, "DFT precision mode must be 0, 1 or 2");
  clarity::set_dft_precision(mode);
  return CLARITY_SUCCESS;
}

int clarityx_dft_precision(void) { return clarity::dft_precision(); }

void clarityx_autotune(int on) {
  std::lock_guard<std::mutex> lk(g_mu);
  g_autotune = on != 0;
  if (g_ctx) {
    std::lock_guard<std::mutex> lk2(g_ctx->mu);
    g_ctx->set_autotune(g_autotune);
  }
}

ClarityResult_t clarityx_blind_ml_device(const float* image, Clarity_Dim3 imageDim,
                                         const float* kernel, Clarity_Dim3 kernelDim,
                                         float* out, int iterations, void* stream) {
  return device_call(image, imageDim, kernel, kernelDim, out, stream,
                     [&](Context& c, const float* i, Dims id, const float* k, Dims kd,
                         float* o) {
                       return clarity::run_blind(c, i, id, k, kd, o, iterations);
                     });
}

ClarityResult_t clarityx_jvc_device(const float* image, Clarity_Dim3 imageDim,
                                    const float* kernel, Clarity_Dim3 kernelDim,
                                    float* out, int iterations, void* stream) {
  return device_call(image, imageDim, kernel, kernelDim, out, stream,
                     [&](Context& c, const float* i, Dims id, const float* k, Dims kd,
                         float* o) {
                       return clarity::run_jvc(c, i, id, k, kd, o, iterations, 0.f,
                                               nullptr, 0);
                     });
}

ClarityResult_t clarityx_idivergence(const float* g, const float* ghat, long long n,
                                     double* result) {
  if (!g || !ghat || !result) return fail(CLARITY_INVALID_ARGUMENT, "NULL buffer");
  if (n <= 0) return fail(CLARITY_INVALID_ARGUMENT, "n <= 0");
  ClarityResult_t rc_ = CLARITY_SUCCESS;
  Context* ctx = acquire_context(&rc_);
  if (!ctx) return rc_;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device());
  ctx->clear_stream();
  float *dg = nullptr, *dh = nullptr;
  cudaError_t e = clarity::dev_alloc((void**)&dg, sizeof(float) * n);
  if (e == cudaSuccess) e = clarity::dev_alloc((void**)&dh, sizeof(float) * n);
  cudaStream_t st = ctx->exec_stream();
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(dg, g, sizeof(float) * n, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(dh, ghat, sizeof(float) * n, cudaMemcpyHostToDevice, st);
  Status s = (e == cudaSuccess) ? clarity::run_idivergence(*ctx, dg, dh, n, result)
                                : clarity::status_from_cuda(e, "idivergence staging");
  cudaFree(dg);
  cudaFree(dh);
  return report(s);
}

ClarityResult_t clarityx_plan_info(Clarity_Dim3 w, int* f, int nf) {
  if (!f || nf <= 0) return fail(CLARITY_INVALID_ARGUMENT, "NULL fields");
  if (!dims_ok(w)) return fail(CLARITY_INVALID_ARGUMENT, "dimension <= 0");
  clarity::VolPlan P;
  std::string why;
  if (!clarity::make_plan(w.x, w.y, w.z, &P, &why))
    return fail(CLARITY_INVALID_ARGUMENT, why);
  const int v[16] = {P.M, P.XS, P.Ay, P.By, P.G, P.W, P.KG, P.xy_blocks, P.z_blocks,
                     P.xy_smem, P.z_smem, P.ax.npass, P.ayB.npass, P.az.npass,
                     P.xmode, (int)(P.spec_elems / 1024)};
  for (int i = 0; i < nf && i < 16; ++i) f[i] = v[i];
  return CLARITY_SUCCESS;
}

}  // extern "C"

// ----------------------------------------------------- benchmark probes
extern "C" {

CLARITY_API long long clarityx_launch_count(void) { return clarity::launch_count(); }

CLARITY_API void clarityx_timing_enable(int on) { clarity::timing_enable(on != 0); }

CLARITY_API void clarityx_timing_collect(double* ms, long long* counts, int n) {
  double m[clarity::KK_COUNT];
  long long c[clarity::KK_COUNT];
  clarity::timing_collect(m, c);
  for (int i = 0; i < n && i < clarity::KK_COUNT; ++i) {
    if (ms) ms[i] = m[i];
    if (counts) counts[i] = c[i];
  }
}

}  // extern "C"
