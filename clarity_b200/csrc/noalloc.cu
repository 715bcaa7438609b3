// noalloc.cu -- circular convolution on device buffers that allocates no
// memory at all (clarityx_convolve_noalloc, include/clarity_ext.h).
//
// Why it exists: some callers must not allocate device memory once they are
// running -- code that runs under a memory pool it manages itself (a
// cudaMalloc behind the pool's back breaks its accounting), real-time loops
// whose memory use must be fixed up front (an allocation can stall or fail
// mid-run), and plugins hosted inside another process's CUDA context that
// forbids cudaMalloc.  The regular entry points allocate their spectra
// and plan tables on first use; this one keeps every scratch buffer (OTF,
// work spectrum, twiddle and digit-reversal tables) in one file-scope
// __device__ array of kScratchBytes.  Every GPU that loads the library holds
// that array until the process exits.
//
// The computation is the one Clarity_Convolve performs (src/Convolve.cxx
// :41-115,146-184), with the same fused kernels as clarityx_convolve_device.
#include <cstdio>
#include <mutex>

#include "../../include/clarity_ext.h"
#include "engine.hpp"
#include "launch_macro.cuh"
#include "ops.cuh"
#include "passes.cuh"
#include "plan.hpp"

namespace clarity {
CLARITY_EXTERN_PASS_KERNELS
namespace {

// 32 MiB: the plan tables, the OTF and the work spectrum.  The limit is in
// bytes, not in a box shape: a work box fits when its two spectra
// (2 x spec_elems x 8 bytes, spec_elems from clarityx_plan_info) and tables
// do -- 128 x 128 x 128 (16.5 MiB) and 128 x 128 x 192 (24.4 MiB) fit,
// 256 x 256 x 256 does not.
constexpr size_t kScratchBytes = size_t(32) << 20;
__device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_addr_mu;
void* g_addr[kMaxDevices] = {};

struct Tables {
  TwTable t[kPlanTwTables];
};

// Twiddles in FP64 (sincospi), rounded; the digit-reversed x slot table.  The
// tables are the planner's own (plan_twiddle_tables, xrev_slot), as the
// cached plans of the other entry points build them.
__global__ void k_noalloc_tables(float2* tw, Tables tabs, int* xrev, AxisPlan ax,
                                 int M) {
  const int stride = gridDim.x * blockDim.x;
  const int t0 = blockIdx.x * blockDim.x + threadIdx.x;
  for (int k = 0; k < kPlanTwTables; ++k) {
    const TwTable T = tabs.t[k];
    for (int t = t0; t < T.count; t += stride) {
      double s, c;
      sincospi(2.0 * (double)t / (double)T.n, &s, &c);
      tw[T.off + t] = make_float2((float)c, (float)(-s));
    }
  }
  for (int k = t0; k < M; k += stride) xrev[k] = xrev_slot(ax, k);
}

size_t round256(size_t v) { return (v + 255) & ~size_t(255); }

ClarityResult_t fail(ClarityResult_t code, const char* msg) {
  set_last_error(msg);
  return code;
}

// Device address of the scratch array on the current device.  In host code
// the array's name is only a host-side stand-in, not a device address, so
// the first call on each device looks the address up (cudaGetSymbolAddress)
// with that device current and keeps it for the life of the process.  That
// first call should therefore come before any stream capture, and the entry
// point must not be used after cudaDeviceReset (which would invalidate the
// kept address).
cudaError_t scratch_address(void** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(g_addr_mu);
  if (!g_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_addr[dev] = p;
  }
  *out = g_addr[dev];
  return cudaSuccess;
}

template <class K>
cudaError_t allow_smem(K kernel, int smem) {
  if (smem > 48 * 1024)
    return cudaFuncSetAttribute(reinterpret_cast<const void*>(kernel),
                                cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  return cudaSuccess;
}

}  // namespace
}  // namespace clarity

using namespace clarity;

extern "C" CLARITY_API ClarityResult_t clarityx_convolve_noalloc(
    const float* image, Clarity_Dim3 imageDim, const float* kernel,
    Clarity_Dim3 kernelDim, float* out, void* stream) {
  if (!image || !kernel || !out) return fail(CLARITY_INVALID_ARGUMENT, "NULL buffer");
  if (imageDim.x <= 0 || imageDim.y <= 0 || imageDim.z <= 0 || kernelDim.x <= 0 ||
      kernelDim.y <= 0 || kernelDim.z <= 0)
    return fail(CLARITY_INVALID_ARGUMENT, "dimension <= 0");
  const int nx = imageDim.x + kernelDim.x, ny = imageDim.y + kernelDim.y,
            nz = imageDim.z + kernelDim.z;
  VolPlan P;
  if (!make_plan(nx, ny, nz, &P, nullptr))
    return fail(CLARITY_INVALID_ARGUMENT, "unsupported work box for the FFT planner");
  // scratch layout: twiddles | x slot table | OTF | work spectrum
  const size_t off_tw = 0;
  const size_t off_rev = round256(off_tw + sizeof(float2) * (size_t)P.twiddle_count);
  const size_t off_h = round256(off_rev + sizeof(int) * (size_t)(P.M > 0 ? P.M : 1));
  const size_t spec_bytes = round256(sizeof(float2) * (size_t)P.spec_elems);
  const size_t off_s = off_h + spec_bytes;
  const size_t need = off_s + spec_bytes;
  if (need > kScratchBytes) {
    char msg[160];
    std::snprintf(msg, sizeof(msg),
                  "work box %dx%dx%d needs %zu bytes of scratch; the no-allocation "
                  "entry point holds %zu",
                  nx, ny, nz, need, kScratchBytes);
    return fail(CLARITY_INVALID_ARGUMENT, msg);
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  void* base = nullptr;
  cudaError_t e = scratch_address(&base);
  if (e != cudaSuccess) return fail(CLARITY_INVALID_OPERATION, cudaGetErrorString(e));
  unsigned char* sc = static_cast<unsigned char*>(base);
  float2* tw = reinterpret_cast<float2*>(sc + off_tw);
  int* xrev = reinterpret_cast<int*>(sc + off_rev);
  float2* H = reinterpret_cast<float2*>(sc + off_h);
  float2* S = reinterpret_cast<float2*>(sc + off_s);

  Tables tabs;
  plan_twiddle_tables(P, tabs.t);
  CLARITY_LAUNCH(k_noalloc_tables, 64, 256, 0, st)(tw, tabs, xrev, P.ax, P.M);

  const Dims wd{nx, ny, nz};
  PaddedSrc pk;
  pk.src = kernel;
  pk.X = kernelDim.x; pk.Y = kernelDim.y; pk.Z = kernelDim.z;
  pk.sx = -kernelDim.x / 2; pk.sy = -kernelDim.y / 2; pk.sz = -kernelDim.z / 2;
  pk.nx = nx; pk.ny = ny; pk.nz = nz;
  const ProPadded pro_k{pk, nullptr, P.xmode};
  const ProImage pro_i{ImageSrc{image, imageDim.x, imageDim.y, imageDim.z}, P.xmode};
  const ModOTF mod{H, 1.0f / ((float)wd.z * wd.y * wd.x)};
  const EpiClip epi{out, imageDim.x, imageDim.y, imageDim.z, nullptr, P.xmode};

  auto kf = k_xy_forward<ProPadded>;
  auto kfi = k_xy_forward<ProImage>;
  auto kzf = k_z<ModForward>;
  auto kzm = k_z<ModOTF>;
  auto ki = k_xy_inverse<EpiClip>;
  if ((e = allow_smem(kf, P.xy_smem)) != cudaSuccess ||
      (e = allow_smem(kfi, P.xy_smem)) != cudaSuccess ||
      (e = allow_smem(kzf, P.z_smem)) != cudaSuccess ||
      (e = allow_smem(kzm, P.z_smem)) != cudaSuccess ||
      (e = allow_smem(ki, P.xy_smem)) != cudaSuccess)
    return fail(CLARITY_INVALID_OPERATION, cudaGetErrorString(e));
  // OTF of the shifted kernel, then R2C(image) * OTF / N, then C2R + clip
  CLARITY_LAUNCH(kf, P.xy_blocks, P.xy_threads, P.xy_smem, st)(P, pro_k, H, tw, xrev);
  CLARITY_LAUNCH(kzf, P.z_blocks, P.z_threads, P.z_smem, st)(P, ModForward{}, H, H, tw);
  CLARITY_LAUNCH(kfi, P.xy_blocks, P.xy_threads, P.xy_smem, st)(P, pro_i, S, tw, xrev);
  CLARITY_LAUNCH(kzm, P.z_blocks, P.z_threads, P.z_smem, st)(P, mod, S, S, tw);
  CLARITY_LAUNCH(ki, P.xy_blocks, P.xy_threads, P.xy_smem, st)(P, epi, S, tw, xrev);
  e = cudaGetLastError();
  if (e != cudaSuccess) return fail(CLARITY_INVALID_OPERATION, cudaGetErrorString(e));
  return CLARITY_SUCCESS;
}
