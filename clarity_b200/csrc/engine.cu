// engine.cu -- planner, device context and the deconvolution algorithms of
// the Clarity path on sm_100a.
//
// Reference: the per-algorithm drivers src/MaximumLikelihoodDeconvolve.cxx
// :160-250, src/WienerDeconvolve.cxx:130-206,
// src/JansenVanCittertDeconvolve.cxx:199-307, src/Convolve.cxx:41-115 and
// src/BlindMaximumLikelihoodDeconvolve.cxx:102-148, which allocate, plan and
// free on every call and synchronise after every kernel.  Here plans and
// buffers are cached per work box, every step is a fused FFT pass, and an
// RL iteration is five kernel launches with no host round trip.
#include <algorithm>
#include <atomic>
#include <climits>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#ifndef CLARITY_HOST_EMULATION
#include <cudaTypedefs.h>
#endif
#include "engine.hpp"
#include "launch.cuh"
#include "ops.cuh"
#include "passes.cuh"

namespace clarity {

#define CL_TRY(expr)              \
  do {                            \
    Status s_ = (expr);           \
    if (!s_.ok()) return s_;      \
  } while (0)

// ------------------------------------------------------------------ errors
Status status_from_cuda(cudaError_t e, const char* what) {
  Status s;
  if (e == cudaSuccess) return s;
  s.code = (e == cudaErrorMemoryAllocation) ? CLARITY_DEVICE_OUT_OF_MEMORY
                                            : CLARITY_INVALID_OPERATION;
  s.msg = std::string(what) + ": " + cudaGetErrorString(e);
  return s;
}


static std::atomic<int> g_alloc_fail_countdown{0};

void set_alloc_failure_countdown(int n) { g_alloc_fail_countdown.store(n); }

cudaError_t dev_alloc(void** p, size_t bytes) {
  int c = g_alloc_fail_countdown.load();
  if (c > 0) {
    if (g_alloc_fail_countdown.fetch_sub(1) == 1) {
      *p = nullptr;
      return cudaErrorMemoryAllocation;  // injected on the host
    }
  }
  return cudaMalloc(p, bytes ? bytes : 16);
}

// ------------------------------------------------------- launch accounting
static std::atomic<long long> g_launches{0};
static std::atomic<bool> g_timing{false};
static std::mutex g_timing_mu;
struct EventPair {
  int kind;
  cudaEvent_t a, b;
};
static std::vector<EventPair> g_events;   // recorded pairs
static std::vector<cudaEvent_t> g_event_pool;
static cudaEvent_t g_pending[KK_COUNT];

static cudaEvent_t take_event() {
  if (!g_event_pool.empty()) {
    cudaEvent_t e = g_event_pool.back();
    g_event_pool.pop_back();
    return e;
  }
  cudaEvent_t e;
  cudaEventCreate(&e);
  return e;
}

// Set while a batch is captured into a graph: launches are counted, but no
// timing events are recorded into the capture.
static thread_local bool t_capturing = false;
void set_capturing(bool on) { t_capturing = on; }
// Programmatic dependent launch of the steady RL passes: off while a graph is
// captured and when CLARITY_PDL=0.
bool pdl_enabled() {
  static const bool on = [] {
    const char* v = std::getenv("CLARITY_PDL");
    return !(v && v[0] == '0');
  }();
  return on && !t_capturing;
}

void note_launch_begin(int kind, cudaStream_t st) {
  g_launches.fetch_add(1);
  if (!g_timing.load() || t_capturing) return;
  std::lock_guard<std::mutex> lk(g_timing_mu);
  cudaEvent_t e = take_event();
  cudaEventRecord(e, st);
  g_pending[kind] = e;
}

void note_launch_end(int kind, cudaStream_t st) {
  if (!g_timing.load() || t_capturing) return;
  std::lock_guard<std::mutex> lk(g_timing_mu);
  cudaEvent_t e = take_event();
  cudaEventRecord(e, st);
  g_events.push_back(EventPair{kind, g_pending[kind], e});
}

long long launch_count() { return g_launches.load(); }

int static_family_mask() {
  static const int mask = [] {
    const char* v = std::getenv("CLARITY_STATIC");
    return v ? std::atoi(v) : 0xF;
  }();
  return mask;
}

static inline void count_small() { g_launches.fetch_add(1); }
void count_launch() { count_small(); }

static std::atomic<int> g_dft_precision{0};
void set_dft_precision(int mode) { g_dft_precision.store(mode); }
int dft_precision() { return g_dft_precision.load(); }

cudaError_t smem_opt_in(const void* kernel, int smem) {
  if (smem <= 48 * 1024) return cudaSuccess;
  static std::mutex mu;
  static std::map<std::pair<const void*, int>, int> done;  // (kernel, device) -> bytes
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(mu);
  int& have = done[{kernel, dev}];
  if (have >= smem) return cudaSuccess;
  const cudaError_t e =
      cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e == cudaSuccess) have = smem;
  return e;
}

bool xy_tma_enabled() {
  static const bool on = [] {
    const char* v = std::getenv("CLARITY_XY_TMA");
    return !(v && v[0] == '0');
  }();
  return on;
}

#ifndef CLARITY_HOST_EMULATION
// cuTensorMapEncodeTiled, fetched from the driver through the runtime (no
// link-time dependency on libcuda).
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 encode = [] {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      fn = nullptr;
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  }();
  return encode;
}
static bool encode_4d(TensorMap* tm, CUtensorMapDataType type, const void* base,
                      const unsigned long long dim[4], const unsigned long long stride_bytes[3],
                      const unsigned box[4], CUtensorMapSwizzle swizzle) {
  PFN_cuTensorMapEncodeTiled_v12000 encode = tensor_map_encoder();
  if (!encode || ((uintptr_t)base & 15u) != 0) return false;
  const cuuint64_t gdim[4] = {dim[0], dim[1], dim[2], dim[3]};
  const cuuint64_t gstr[3] = {stride_bytes[0], stride_bytes[1], stride_bytes[2]};
  const cuuint32_t bdim[4] = {box[0], box[1], box[2], box[3]};
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  return encode(tm, type, 4, const_cast<void*>(base), gdim, gstr, bdim, estr,
                CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}
bool encode_tensor_f32_4d(TensorMap* tm, const void* base, const unsigned long long dim[4],
                          const unsigned long long stride_bytes[3], const unsigned box[4]) {
  return encode_4d(tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, base, dim, stride_bytes, box,
                   CU_TENSOR_MAP_SWIZZLE_NONE);
}
bool encode_tensor_bf16_4d(TensorMap* tm, const void* base, const unsigned long long dim[4],
                           const unsigned long long stride_bytes[3], const unsigned box[4],
                           bool swizzle32) {
  return encode_4d(tm, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, base, dim, stride_bytes, box,
                   swizzle32 ? CU_TENSOR_MAP_SWIZZLE_32B : CU_TENSOR_MAP_SWIZZLE_NONE);
}
#else
bool encode_tensor_f32_4d(TensorMap* tm, const void* base, const unsigned long long dim[4],
                          const unsigned long long stride_bytes[3], const unsigned box[4]) {
  if (((uintptr_t)base & 15u) != 0) return false;
  tm->base = static_cast<char*>(const_cast<void*>(base));
  for (int d = 0; d < 4; ++d) {
    tm->dim[d] = dim[d];
    tm->box[d] = box[d];
    tm->stride[d] = d == 0 ? 4 : stride_bytes[d - 1];
  }
  return true;
}
#endif

void timing_enable(bool on) { g_timing.store(on); }

void timing_collect(double* ms, long long* counts) {
  std::lock_guard<std::mutex> lk(g_timing_mu);
  for (int k = 0; k < KK_COUNT; ++k) { ms[k] = 0; counts[k] = 0; }
  for (auto& p : g_events) {
    cudaEventSynchronize(p.b);
    float t = 0;
    cudaEventElapsedTime(&t, p.a, p.b);
    ms[p.kind] += t;
    counts[p.kind] += 1;
    g_event_pool.push_back(p.a);
    g_event_pool.push_back(p.b);
  }
  g_events.clear();
}

// ------------------------------------------------------------ small kernels
// w_n^t = exp(-2 pi i t / n), evaluated in FP64 with sincospi and rounded.
__global__ void k_gen_twiddles(float2* tw, const TwTable* tabs, int ntab) {
  for (int k = 0; k < ntab; ++k) {
    const TwTable T = tabs[k];
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < T.count;
         t += gridDim.x * blockDim.x) {
      double s, c;
      sincospi(2.0 * (double)t / (double)T.n, &s, &c);
      tw[T.off + t] = make_float2((float)c, (float)(-s));
    }
  }
}

// FP64 partial sums of a float array (grid-stride; fixed grid -> fixed order).
__global__ void k_reduce_sum(const float* __restrict__ a, long long n,
                             double* __restrict__ partial) {
  double acc = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    acc += (double)a[i];
  block_sum_store(acc, partial);
}


// sum -> dout[0]
__global__ void k_finish_sum(const double* partial, int np, double* dout) {
  const double t = block_total(partial, np);
  if (threadIdx.x == 0) dout[0] = t;
}

// The image on the work box (zero padding), as the first RL estimate.
__global__ void k_pad_image(ImageSrc g, WorkVol w, float* __restrict__ out) {
  const long long n = (long long)w.nx * w.ny * w.nz;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % w.nx);
    const long long r = i / w.nx;
    out[i] = g.at(x, (int)(r % w.ny), (int)(r / w.ny));
  }
}

// Accelerated RL step bookkeeping: x_next = s u' (in place over u'),
// g_k = x_next - y, and (after the first step) FP64 sums of g_k g_{k-1} and
// g_{k-1}^2 per block into partial[2b], partial[2b+1]; g_{k-1} is replaced by
// g_k.
__global__ void k_accel_update(float* __restrict__ u, const float* __restrict__ y,
                               float* __restrict__ gprev, const float* __restrict__ scale,
                               int first, long long n, double* __restrict__ partial) {
  const float s = *scale;
  double d1 = 0, d2 = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const float v = s * u[i];
    const float g = v - y[i];
    if (!first) {
      const float gp = gprev[i];
      d1 += (double)g * (double)gp;
      d2 += (double)gp * (double)gp;
    }
    gprev[i] = g;
    u[i] = v;
  }
  block_sum_store(d1, partial + 0 * gridDim.x);
  block_sum_store(d2, partial + 1 * gridDim.x);
}

// alpha = sum(g_k g_{k-1}) / sum(g_{k-1}^2) clamped to [0, 1], as float.
__global__ void k_finish_alpha(const double* partial, int np, float* alpha) {
  const double a = block_total(partial, np);
  __syncthreads();
  const double b = block_total(partial + np, np);
  if (threadIdx.x == 0) {
    float r = 0.f;
    if (b > 0) {
      r = (float)(a / b);
      r = r < 0.f ? 0.f : (r > 1.f ? 1.f : r);
    }
    *alpha = r;
  }
}

// sum of *np partials -> *dout (the count is written by the producing pass)
__global__ void k_finish_sum_np(const double* partial, const int* np, double* dout) {
  const double t = block_total(partial, *np);
  if (threadIdx.x == 0) dout[0] = t;
}

// RL flux scale (src/MaximumLikelihoodDeconvolve.cxx:73-78):
// scale = energy / newEnergy with both rounded to float first, as the
// reference holds them in floats.  It runs once per RL iteration on the
// critical path between two passes, so a full 1024-thread block reads the
// partials (4096 at the 512x512x128 box: four per thread); block_total
// handles up to 32 warps.
static constexpr int kFinishThreads = 1024;
__global__ void __launch_bounds__(kFinishThreads)
    k_finish_rl_scale(const double* partial, const int* np, const double* energy,
                      double* sum_out, float* scale_out) {
  CLARITY_PDL_WAIT();  // the product pass's partials are complete and visible
  const double t = block_total(partial, *np);
  if (threadIdx.x == 0) {
    sum_out[0] = t;
    scale_out[0] = (float)energy[0] / (float)t;
  }
}

// 1 / sum, in float (Clarity_NormalizeArray, src/ComputePrimitives.cxx:197-209)
__global__ void k_finish_inverse(const double* partial, int np, float* out) {
  const double t = block_total(partial, np);
  if (threadIdx.x == 0) out[0] = 1.0f / (float)t;
}

// Crop the work box to the image region, times an optional device scale.
__global__ void k_clip(const float* __restrict__ w, int nx, int ny,
                       float* __restrict__ out, int X, int Y, int Z,
                       const float* __restrict__ scale) {
  const long long n = (long long)X * Y * Z;
  const float s = scale ? *scale : 1.f;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % X);
    const long long r = i / X;
    const int y = (int)(r % Y);
    const int z = (int)(r / Y);
    const float v = w[((long long)z * ny + y) * nx + x];
    out[i] = scale ? s * v : v;
  }
}

__global__ void k_copy(const float* __restrict__ a, float* __restrict__ b,
                       long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    b[i] = a[i];
}

static constexpr int kReduceBlocks = 592;  // 4 x 148 SMs

// hc = conj(h) over a spectrum: the OTF of the reflected kernel h(-x), whose
// product is a correlation with h.
__global__ void k_conj_spectrum(const float2* __restrict__ h, float2* __restrict__ hc,
                                long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const float2 v = h[i];
    hc[i] = make_float2(v.x, -v.y);
  }
}

// uint16 raw volumes (the reference's DeconvolveRawImages app,
// apps/DeconvolveRawImages/DeconvolveRawImages.cxx:91-116): cast in, and cast
// out as x86 does for static_cast<unsigned short>(float) -- truncation to a
// 32-bit integer (0x80000000 for NaN and |x| >= 2^31), low 16 bits kept.
__global__ void k_u16_to_f32(const uint16_t* __restrict__ a, float* __restrict__ b, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    b[i] = (float)a[i];
}
__global__ void k_f32_to_u16(const float* __restrict__ a, uint16_t* __restrict__ b, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const float x = a[i];
    const int v = (fabsf(x) < 2147483648.f) ? __float2int_rz(x) : INT_MIN;  // NaN fails the test
    b[i] = (uint16_t)((unsigned)v & 0xFFFFu);
  }
}

Status cast_u16_to_f32(Context& ctx, const uint16_t* a, float* b, long long n) {
  count_small();
  CLARITY_LAUNCH(k_u16_to_f32, kReduceBlocks, 256, 0, ctx.exec_stream())(a, b, n);
  CL_CHECK(cudaGetLastError());
  return Status::Ok();
}
Status cast_f32_to_u16(Context& ctx, const float* a, uint16_t* b, long long n) {
  count_small();
  CLARITY_LAUNCH(k_f32_to_u16, kReduceBlocks, 256, 0, ctx.exec_stream())(a, b, n);
  CL_CHECK(cudaGetLastError());
  return Status::Ok();
}

// max of a float array: block maxima then a single-block finish.
__global__ void k_reduce_max(const float* __restrict__ a, long long n,
                             float* __restrict__ partial) {
  float m = -INFINITY;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    m = fmaxf(m, a[i]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  __shared__ float red[32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = red[0];
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) t = fmaxf(t, red[w]);
    partial[blockIdx.x] = t;
  }
}

// JVC constants from the image maximum (src/JansenVanCittertDeconvolve.cxx
// :128-129): A = 0.5 max, invASq = 1 / (A A).  out[0] = A, out[1] = invASq.
__global__ void k_finish_jvc(const float* partial, int np, float* out) {
  if (threadIdx.x == 0) {
    float m = partial[0];
    for (int i = 1; i < np; ++i) m = fmaxf(m, partial[i]);
    const float A = 0.5f * m;
    out[0] = A;
    out[1] = 1.0f / (A * A);
  }
}

// I-divergence partials: g ln(g/ghat) + ghat - g (0 ln 0 = 0), FP64.
__global__ void k_idiv(const float* __restrict__ g, const float* __restrict__ gh,
                       long long n, double* __restrict__ partial) {
  double acc = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const double a = g[i], b = gh[i];
    if (a > 0) {
      if (b > 0) acc += a * log(a / b) + b - a;
    } else {
      acc += b - a;
    }
  }
  block_sum_store(acc, partial);
}


// --------------------------------------------------------------- context
Context::Context(int device) : device_(device) {}

Status Context::init() {
  CL_CHECK(cudaSetDevice(device_));
  CL_CHECK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
  void* h = nullptr;
  CL_CHECK(cudaHostAlloc(&h, sizeof(int), cudaHostAllocMapped | cudaHostAllocPortable));
  err_host_ = static_cast<int*>(h);
  *reinterpret_cast<volatile int*>(err_host_) = 0;
  void* d = nullptr;
  CL_CHECK(cudaHostGetDevicePointer(&d, h, 0));
  err_dev_ = static_cast<int*>(d);
  return Status::Ok();
}

Context::~Context() {
  cudaSetDevice(device_);
  release_workspaces();
  for (cudaStream_t b : bstreams_) cudaStreamDestroy(b);
  bstreams_.clear();
  for (auto& kv : plans_) {
    cudaFree(kv.second->tw);
    cudaFree(kv.second->xrev);
  }
  plans_.clear();
  if (stream_) cudaStreamDestroy(stream_);
  if (err_host_) cudaFreeHost(err_host_);
}

static void free_workspace(Workspace& w) {
  cudaFree(w.S); cudaFree(w.H); cudaFree(w.u); cudaFree(w.img); cudaFree(w.ker);
  cudaFree(w.partial); cudaFree(w.dscal); cudaFree(w.fscal); cudaFree(w.iscal);
  cudaFree(w.HG);
  for (float* b : w.accel) cudaFree(b);
  for (float* b : w.xbuf) cudaFree(b);
  w = Workspace();
}

void Context::release_workspaces() {
  // graphs hold workspace addresses: they go first
  for (auto& g : graphs_) cudaGraphExecDestroy(g.exec);
  graphs_.clear();
  free_workspace(ws_);
  for (auto& w : slots_) free_workspace(*w);
  slots_.clear();
  cudaFree(aux_);
  aux_ = nullptr;
  aux_cap_ = 0;
  cudaFree(bq_);
  bq_ = nullptr;
  bq_cap_ = 0;
}

Status Context::batch_scratch(size_t bytes, void** out) {
  if (bq_cap_ < bytes || !bq_) {
    // graphs captured with the old buffer would use it after it is freed
    cudaStreamSynchronize(stream_);
    for (auto& g : graphs_) cudaGraphExecDestroy(g.exec);
    graphs_.clear();
    cudaFree(bq_);
    bq_ = nullptr;
    bq_cap_ = 0;
    CL_CHECK(dev_alloc(&bq_, bytes));
    bq_cap_ = bytes;
  }
  *out = bq_;
  return Status::Ok();
}

Status Context::aux_scratch(size_t bytes, void** out) {
  if (aux_cap_ < bytes || !aux_) {
    cudaFree(aux_);
    aux_ = nullptr;
    aux_cap_ = 0;
    CL_CHECK(dev_alloc(&aux_, bytes));
    aux_cap_ = bytes;
  }
  *out = aux_;
  return Status::Ok();
}

Status Context::batch_stream(int i, cudaStream_t* out) {
  while ((int)bstreams_.size() <= i) {
    cudaStream_t b = nullptr;
    CL_CHECK(cudaStreamCreateWithFlags(&b, cudaStreamNonBlocking));
    bstreams_.push_back(b);
  }
  *out = bstreams_[i];
  return Status::Ok();
}

cudaGraphExec_t Context::find_graph(const std::vector<unsigned long long>& key) const {
  for (const auto& g : graphs_)
    if (g.key == key) return g.exec;
  return nullptr;
}

void Context::add_graph(std::vector<unsigned long long> key, cudaGraphExec_t g) {
  constexpr size_t kMaxGraphs = 8;  // oldest first out
  if (graphs_.size() >= kMaxGraphs) {
    cudaGraphExecDestroy(graphs_.front().exec);
    graphs_.erase(graphs_.begin());
  }
  graphs_.push_back(GraphEntry{std::move(key), g});
}

Status Context::build_entry(const VolPlan& P0, std::unique_ptr<PlanEntry>* out) {
  auto pe = std::make_unique<PlanEntry>();
  pe->P = P0;
  const VolPlan& P = pe->P;
  CL_CHECK(dev_alloc((void**)&pe->tw, sizeof(float2) * P.twiddle_count));
  CL_CHECK(dev_alloc((void**)&pe->xrev, sizeof(int) * std::max(P.xrev_count, 1)));
  pe->err = err_dev_;
  std::vector<int> rev;
  std::vector<TwTable> tabs;
  plan_tables(P, &rev, &tabs);
  TwTable* dtabs = nullptr;
  CL_CHECK(dev_alloc((void**)&dtabs, sizeof(TwTable) * tabs.size()));
  cudaStream_t st = exec_stream();
  CL_CHECK(cudaMemcpyAsync(pe->xrev, rev.data(), sizeof(int) * rev.size(),
                           cudaMemcpyHostToDevice, st));
  CL_CHECK(cudaMemcpyAsync(dtabs, tabs.data(), sizeof(TwTable) * tabs.size(),
                           cudaMemcpyHostToDevice, st));
  CLARITY_LAUNCH(k_gen_twiddles, 64, 256, 0, st)(pe->tw, dtabs, (int)tabs.size());
  CL_CHECK(cudaGetLastError());
  CL_CHECK(cudaStreamSynchronize(st));
  cudaFree(dtabs);
  *out = std::move(pe);
  return Status::Ok();
}

static void free_entry(PlanEntry& pe) {
  cudaFree(pe.tw);
  cudaFree(pe.xrev);
}

Status Context::plan(const Dims& wd, const PlanEntry** out) {
  // tuned and default plans are cached apart: a plan the autotuner picked
  // (by timings that vary from run to run) must not serve calls made with
  // autotuning off, or results would depend on what ran before
  auto key = std::make_tuple(wd.x, wd.y, wd.z, autotune_ ? 1 : 0);
  auto it = plans_.find(key);
  if (it != plans_.end()) {
    *out = it->second.get();
    return Status::Ok();
  }
  std::unique_ptr<PlanEntry> pe;
  if (autotune_) {
    CL_TRY(tune(wd, &pe));
  } else {
    VolPlan P;
    std::string why;
    if (!make_plan(wd.x, wd.y, wd.z, &P, &why)) {
      Status s;
      s.code = CLARITY_INVALID_ARGUMENT;
      s.msg = "unsupported work box " + std::to_string(wd.x) + "x" +
              std::to_string(wd.y) + "x" + std::to_string(wd.z) + ": " + why;
      return s;
    }
    CL_TRY(build_entry(P, &pe));
  }
  *out = pe.get();
  plans_[key] = std::move(pe);
  return Status::Ok();
}

Status Context::check_device_errors() {
  if (!err_host_) return Status::Ok();
  const int e = __atomic_exchange_n(err_host_, 0, __ATOMIC_ACQ_REL);
  if (e == 0) return Status::Ok();
  Status s;
  s.code = CLARITY_INVALID_OPERATION;
  s.msg = e == kErrWaitTimeout
              ? "a device-side wait timed out; the result of the call that ran it is not valid"
              : "a device-side copy address was misaligned (code " + std::to_string(e) +
                    "); the result of the call that ran it is not valid";
  return s;
}

// Failure-detection self test: one thread arms an mbarrier for 16 bytes that
// no copy will ever deliver and waits on it with a bound of `limit` polls,
// exactly as a fused pass waits for its tile.  The wait gives up and records
// kErrWaitTimeout in the error word.  No copy is issued, so nothing is left
// in flight when the block exits.
__global__ void k_wait_timeout_probe(int* err, long long limit) {
  __shared__ alignas(8) uint64_t bar;
  if (threadIdx.x != 0) return;
  mbar_init(&bar, 1);
  mbar_arrive_expect_tx(&bar, 16);
  mbar_wait_bounded(&bar, 0, err, limit);
}

Status inject_wait_timeout(Context& ctx) {
  count_small();
  CLARITY_LAUNCH(k_wait_timeout_probe, 1, 32, 0, ctx.exec_stream())(ctx.err_dev(), 1ll << 14);
  CL_CHECK(cudaGetLastError());
  return Status::Ok();
}

template <class T>
static Status ensure(T** p, long long* cap, long long need) {
  if (*cap >= need && *p) return Status::Ok();
  cudaFree(*p);
  *p = nullptr;
  *cap = 0;
  CL_CHECK(dev_alloc((void**)p, sizeof(T) * (size_t)need));
  *cap = need;
  return Status::Ok();
}

// A set of work-box volumes of at least n floats each (reallocated together).
template <int K>
static Status ensure_volumes(float* (&bufs)[K], long long* cap, long long n) {
  if (*cap >= n) return Status::Ok();
  for (float*& b : bufs) {
    cudaFree(b);
    b = nullptr;
  }
  *cap = 0;
  for (float*& b : bufs) CL_CHECK(dev_alloc((void**)&b, sizeof(float) * (size_t)n));
  *cap = n;
  return Status::Ok();
}

static Status fill_workspace(Workspace& w, const PlanEntry& pe, const Dims& img,
                             const Dims& ker);

Status Context::workspace(const PlanEntry& pe, const Dims& img, const Dims& ker,
                          Workspace** out) {
  CL_TRY(fill_workspace(ws_, pe, img, ker));
  *out = &ws_;
  return Status::Ok();
}

Status Context::workspace_slot(int slot, const PlanEntry& pe, const Dims& img, const Dims& ker,
                               Workspace** out) {
  while ((int)slots_.size() <= slot) slots_.push_back(std::make_unique<Workspace>());
  CL_TRY(fill_workspace(*slots_[slot], pe, img, ker));
  *out = slots_[slot].get();
  return Status::Ok();
}

static Status fill_workspace(Workspace& w, const PlanEntry& pe, const Dims& img,
                             const Dims& ker) {
  const VolPlan& P = pe.P;
  long long sc = w.spec_cap;
  Status s;
  if (w.spec_cap < P.spec_elems || !w.S || !w.H) {
    cudaFree(w.S); cudaFree(w.H); cudaFree(w.HG);
    w.S = w.H = w.HG = nullptr;
    w.spec_cap = 0;
    CL_CHECK(dev_alloc((void**)&w.S, sizeof(float2) * (size_t)P.spec_elems));
    CL_CHECK(dev_alloc((void**)&w.H, sizeof(float2) * (size_t)P.spec_elems));
    w.spec_cap = P.spec_elems;
  }
  (void)sc;
  s = ensure(&w.u, &w.work_cap, P.n_real());
  if (!s.ok()) return s;
  long long ic = (long long)w.img_cap, kc = (long long)w.ker_cap;
  s = ensure(&w.img, &ic, img.n());
  if (!s.ok()) return s;
  w.img_cap = (size_t)ic;
  s = ensure(&w.ker, &kc, ker.n());
  if (!s.ok()) return s;
  w.ker_cap = (size_t)kc;
  long long pc = w.partial_cap;
  // one partial per XY block: at most one block per (z, y0) line
  s = ensure(&w.partial, &pc,
             std::max<long long>({(long long)P.xy_blocks, (long long)P.nz * P.By,
                                  (long long)kReduceBlocks, 1}));
  if (!s.ok()) return s;
  w.partial_cap = (int)pc;
  if (!w.dscal) CL_CHECK(dev_alloc((void**)&w.dscal, sizeof(double) * 16));
  if (!w.fscal) CL_CHECK(dev_alloc((void**)&w.fscal, sizeof(float) * 16));
  if (!w.iscal) CL_CHECK(dev_alloc((void**)&w.iscal, sizeof(int) * 16));
  return Status::Ok();
}

// Launch wrappers are instantiated in the kern_*.cu translation units.
CLARITY_EXTERN_LAUNCHES


static PaddedSrc padded(const float* src, Dims sd, Dims wd, int sx, int sy,
                        int sz) {
  PaddedSrc p;
  p.src = src;
  p.X = sd.x; p.Y = sd.y; p.Z = sd.z;
  p.sx = sx; p.sy = sy; p.sz = sz;
  p.nx = wd.x; p.ny = wd.y; p.nz = wd.z;
  return p;
}

static ImageSrc image_src(const float* src, Dims sd) {
  return ImageSrc{src, sd.x, sd.y, sd.z};
}

static Dims work_dims(Dims id, Dims kd) {
  return Dims{id.x + kd.x, id.y + kd.y, id.z + kd.z};
}

static float inv_volume(const Dims& wd) {
  // src/Convolve.cxx:199: 1.0f / ((float) nz*ny*nx)
  return 1.0f / ((float)wd.z * wd.y * wd.x);
}

// OTF: R2C of the kernel padded to the work box and shifted by -kernelDim/2
// (src/MaximumLikelihoodDeconvolve.cxx:286-289,181), in the S layout.
static Status make_otf(Context& ctx, const PlanEntry& pe, const float* ker,
                       Dims kd, Dims wd, float2* H, const float* scale) {
  ProPadded pro;
  pro.p = padded(ker, kd, wd, -kd.x / 2, -kd.y / 2, -kd.z / 2);
  pro.scale = scale;
  pro.xmode = pe.P.xmode;
  CL_TRY(xy_forward(ctx, pe, pro, H));
  CL_TRY(z_pass(ctx, pe, ModForward{}, H, H));
  return Status::Ok();
}

static Status setup(Context& ctx, Dims id, Dims kd, const PlanEntry** pe,
                    Workspace** ws, Dims* wd) {
  *wd = work_dims(id, kd);
  CL_TRY(ctx.plan(*wd, pe));
  CL_TRY(ctx.workspace(**pe, id, kd, ws));
  return Status::Ok();
}

static Status reduce_sum_into(Context& ctx, const float* a, long long n,
                              double* partial, double* dout) {
  cudaStream_t st = ctx.exec_stream();
  count_small();
  CLARITY_LAUNCH(k_reduce_sum, kReduceBlocks, 256, 0, st)(a, n, partial);
  count_small();
  CLARITY_LAUNCH(k_finish_sum, 1, 256, 0, st)(partial, kReduceBlocks, dout);
  CL_CHECK(cudaGetLastError());
  return Status::Ok();
}

// Autotuner: builds the planner's best few tilings of the box and times one
// Richardson-Lucy iteration's passes (z, ratio, z, product) with each on
// zero-filled scratch volumes; the fastest plan is kept.
Status Context::tune(const Dims& wd, std::unique_ptr<PlanEntry>* out) {
  VolPlan cand[4];
  std::string why;
  const int nc = make_plan_candidates(wd.x, wd.y, wd.z, cand, 4, &why);
  if (nc == 0) {
    Status s;
    s.code = CLARITY_INVALID_ARGUMENT;
    s.msg = "unsupported work box " + std::to_string(wd.x) + "x" + std::to_string(wd.y) +
            "x" + std::to_string(wd.z) + ": " + why;
    return s;
  }
  if (nc == 1) return build_entry(cand[0], out);
  long long spec = 0, parts = kReduceBlocks;
  for (int c = 0; c < nc; ++c) {
    spec = std::max(spec, cand[c].spec_elems);
    parts = std::max<long long>({parts, (long long)cand[c].xy_blocks,
                                 (long long)cand[c].nz * cand[c].By});
  }
  float2* S = nullptr;
  float* u = nullptr;
  double* partial = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  std::unique_ptr<PlanEntry> best;
  float best_ms = 0.f;
  Status st = Status::Ok();
  cudaStream_t sm = exec_stream();
  auto run = [&]() -> Status {
    CL_CHECK(dev_alloc((void**)&S, sizeof(float2) * (size_t)spec));
    CL_CHECK(dev_alloc((void**)&u, sizeof(float) * (size_t)wd.n()));
    CL_CHECK(dev_alloc((void**)&partial, sizeof(double) * (size_t)parts));
    CL_CHECK(cudaMemsetAsync(S, 0, sizeof(float2) * (size_t)spec, sm));
    CL_CHECK(cudaMemsetAsync(u, 0, sizeof(float) * (size_t)wd.n(), sm));
    CL_CHECK(cudaEventCreate(&e0));
    CL_CHECK(cudaEventCreate(&e1));
    const ImageSrc g{u, wd.x, wd.y, wd.z};
    const WorkVol wv{wd.x, wd.y, wd.z};
    for (int c = 0; c < nc; ++c) {
      std::unique_ptr<PlanEntry> pe;
      CL_TRY(build_entry(cand[c], &pe));
      const int xm = pe->P.xmode;
      auto iteration = [&]() -> Status {
        CL_TRY(z_pass(*this, *pe, ModOTF{S, 1.f}, S, S));
        CL_TRY(xy_inv_fwd(*this, *pe, MidRLRatio{g, xm}, S));
        CL_TRY(z_pass(*this, *pe, ModOTF{S, 1.f}, S, S));
        EpiRLProduct epi{};
        epi.cur = u; epi.g = g; epi.scale = nullptr; epi.unew = u; epi.partial = partial;
        epi.w = wv; epi.xmode = xm; epi.acc = 0.0; epi.nblocks = nullptr;
        CL_TRY(xy_inv_fwd(*this, *pe, epi, S));
        return Status::Ok();
      };
      CL_TRY(iteration());  // warm-up (first launches configure the kernels)
      CL_CHECK(cudaEventRecord(e0, sm));
      for (int r = 0; r < 3; ++r) CL_TRY(iteration());
      CL_CHECK(cudaEventRecord(e1, sm));
      CL_CHECK(cudaEventSynchronize(e1));
      float ms = 0.f;
      CL_CHECK(cudaEventElapsedTime(&ms, e0, e1));
      if (!best || ms < best_ms) {
        if (best) free_entry(*best);
        best = std::move(pe);
        best_ms = ms;
      } else {
        free_entry(*pe);
      }
    }
    return Status::Ok();
  };
  st = run();
  cudaStreamSynchronize(sm);
  cudaFree(S);
  cudaFree(u);
  cudaFree(partial);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (!st.ok()) {
    if (best) free_entry(*best);
    return st;
  }
  *out = std::move(best);
  return Status::Ok();
}

Status run_convolve(Context& ctx, const float* img, Dims id, const float* ker,
                    Dims kd, float* out) {
  const PlanEntry* pe;
  Workspace* ws;
  Dims wd;
  CL_TRY(setup(ctx, id, kd, &pe, &ws, &wd));
  const VolPlan& P = pe->P;
  CL_TRY(make_otf(ctx, *pe, ker, kd, wd, ws->H, nullptr));
  ProImage pro{image_src(img, id), P.xmode};
  CL_TRY(xy_forward(ctx, *pe, pro, ws->S));
  CL_TRY(z_pass(ctx, *pe, ModOTF{ws->H, inv_volume(wd)}, ws->S, ws->S));
  EpiClip epi{out, id.x, id.y, id.z, nullptr, P.xmode};
  CL_TRY(xy_inverse(ctx, *pe, epi, ws->S));
  return Status::Ok();
}

// Circular correlation: Clarity_Convolve's passes with the conjugated OTF
// applied in the z pass.
Status run_correlate(Context& ctx, const float* img, Dims id, const float* ker, Dims kd,
                     float* out) {
  const PlanEntry* pe;
  Workspace* ws;
  Dims wd;
  CL_TRY(setup(ctx, id, kd, &pe, &ws, &wd));
  const VolPlan& P = pe->P;
  CL_TRY(make_otf(ctx, *pe, ker, kd, wd, ws->H, nullptr));
  if (!ws->HG) CL_CHECK(dev_alloc((void**)&ws->HG, sizeof(float2) * (size_t)ws->spec_cap));
  count_small();
  CLARITY_LAUNCH(k_conj_spectrum, kReduceBlocks, 256, 0, ctx.exec_stream())(ws->H, ws->HG,
                                                                            P.spec_elems);
  CL_CHECK(cudaGetLastError());
  ProImage pro{image_src(img, id), P.xmode};
  CL_TRY(xy_forward(ctx, *pe, pro, ws->S));
  CL_TRY(z_pass(ctx, *pe, ModOTF{ws->HG, inv_volume(wd)}, ws->S, ws->S));
  EpiClip epi{out, id.x, id.y, id.z, nullptr, P.xmode};
  CL_TRY(xy_inverse(ctx, *pe, epi, ws->S));
  return Status::Ok();
}

Status run_wiener(Context& ctx, const float* img, Dims id, const float* ker,
                  Dims kd, float* out, float eps) {
  const PlanEntry* pe;
  Workspace* ws;
  Dims wd;
  CL_TRY(setup(ctx, id, kd, &pe, &ws, &wd));
  const VolPlan& P = pe->P;
  CL_TRY(make_otf(ctx, *pe, ker, kd, wd, ws->H, nullptr));
  ProImage pro{image_src(img, id), P.xmode};
  CL_TRY(xy_forward(ctx, *pe, pro, ws->S));
  CL_TRY(z_pass(ctx, *pe, ModWiener{ws->H, eps, inv_volume(wd)}, ws->S, ws->S));
  EpiClip epi{out, id.x, id.y, id.z, nullptr, P.xmode};
  CL_TRY(xy_inverse(ctx, *pe, epi, ws->S));
  return Status::Ok();
}

// Richardson-Lucy (src/MaximumLikelihoodDeconvolve.cxx:48-81), four fused
// passes per iteration after a one-off forward transform of the image:
//   P2 z pass: y0/z forward, * OTF * s/N, inverse        -> S   (h * cur)
//   P3 xy inverse, r = g / (h*cur) with the 1e-5 guard, xy forward -> S
//   P4 z pass again                                      -> S   (h * r)
//   P5 xy inverse, u' = cur * (h*r), FP64 partial sums, and (except on the
//      last iteration) the xy forward transform of u'   -> u, S
// then s = E / sum(u') on the device.  cur = s*u' is never stored: P5 reads
// u' and s, and P2 of the next iteration applies s to the transform of u'
// (the flux rescale of :73-78, deferred).
// start: the first estimate (an image-sized volume, zero in the padding;
// nullptr: the image itself, as the reference).  idiv: when not null,
// idiv[k] (k < iters) receives the I-divergence of the image against
// h * (estimate at the start of iteration k), accumulated by the ratio pass,
// and idiv[iters] that of the result.
//
// Blind ML's alternating updates reuse it with other roles (RLRoles): the OTF
// may be another spectrum (the object's, for the PSF update), the start a
// work-box volume, and the rescale target 1 (the PSF's unit sum) instead of
// the image's energy.
struct RLRoles {
  const float2* otf = nullptr;  // fully transformed OTF (nullptr: ws.H)
  const float2* otf2 = nullptr; // the second convolution's OTF (nullptr: otf)
  Dims start_dims{0, 0, 0};     // start's extent on the work box (0: the image's)
  bool unit_energy = false;     // rescale to sum 1 instead of sum(image)
};

__global__ void k_set_double(double* p, double v) { *p = v; }

// The kernel image on the work box through the reference's pad/shift map,
// times *scale (1 / its sum): the blind update's PSF estimate.
__global__ void k_pad_scaled(PaddedSrc p, const float* __restrict__ scale, float* __restrict__ out) {
  const long long n = (long long)p.nx * p.ny * p.nz;
  const float s = *scale;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % p.nx);
    const long long r = i / p.nx;
    out[i] = s * p.at(x, (int)(r % p.ny), (int)(r / p.ny));
  }
}

// out = *scale * in (work box)
__global__ void k_scale_copy(const float* __restrict__ in, const float* __restrict__ scale,
                             float* __restrict__ out, long long n) {
  const float s = *scale;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    out[i] = s * in[i];
}

// The PSF estimate back on the kernel's own grid: the inverse of the pad/shift
// by -kdim/2, psf[s] = h[(s - kdim/2) mod work dim].
__global__ void k_unpad_psf(const float* __restrict__ h, Dims wd, Dims kd, float* __restrict__ psf) {
  const long long n = (long long)kd.x * kd.y * kd.z;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % kd.x);
    const long long r = i / kd.x;
    const int y = (int)(r % kd.y), z = (int)(r / kd.y);
    const int dx = ((x - kd.x / 2) % wd.x + wd.x) % wd.x;
    const int dy = ((y - kd.y / 2) % wd.y + wd.y) % wd.y;
    const int dz = ((z - kd.z / 2) % wd.z + wd.z) % wd.z;
    psf[i] = h[((long long)dz * wd.y + dy) * wd.x + dx];
  }
}

static Status rl_core(Context& ctx, const PlanEntry& pe, Workspace& ws,
                      const float* img, Dims id, Dims wd, int iters,
                      bool rescale, const float* start = nullptr, double* idiv = nullptr,
                      const RLRoles& roles = RLRoles{}) {
  const VolPlan& P = pe.P;
  cudaStream_t st = ctx.exec_stream();
  const ImageSrc g = image_src(img, id);
  const Dims sd = roles.start_dims.x > 0 ? roles.start_dims : id;
  const ImageSrc u0 = start ? image_src(start, sd) : g;
  const float2* H = roles.otf ? roles.otf : ws.H;
  const float2* H2 = roles.otf2 ? roles.otf2 : H;
  const WorkVol wv{wd.x, wd.y, wd.z};
  const float scale_n = inv_volume(wd);
  float* sdev = ws.fscal;  // deferred flux scale
  if (rescale) {
    if (roles.unit_energy) {
      count_small();
      CLARITY_LAUNCH(k_set_double, 1, 1, 0, st)(ws.dscal + 0, 1.0);
      CL_CHECK(cudaGetLastError());
    } else {
      CL_TRY(reduce_sum_into(ctx, img, id.n(), ws.partial, ws.dscal + 0));
    }
  }
  CL_TRY(xy_forward(ctx, pe, ProImage{u0, P.xmode}, ws.S));
  for (int k = 0; k < iters; ++k) {
    const float* sk = (k == 0 || !rescale) ? nullptr : sdev;
    // P3 reads only planes z < Z (the image is zero beyond): the rest of this
    // pass's output is neither inverse-transformed along y0 nor stored
    ModOTF m2{H, scale_n, sk};
    m2.zout = id.z;
    CL_TRY(z_pass(ctx, pe, m2, ws.S, ws.S));
    MidRLRatio ratio{g, P.xmode};
    if (idiv) {
      ratio.idiv_partial = ws.partial;
      ratio.nblocks = ws.iscal + 1;
    }
    CL_TRY(xy_inv_fwd(ctx, pe, ratio, ws.S));
    if (idiv) {
      // read before the product pass reuses the partials
      count_small();
      CLARITY_LAUNCH(k_finish_sum_np, 1, 256, 0, st)(ws.partial, ws.iscal + 1, idiv + k);
      CL_CHECK(cudaGetLastError());
    }
    // the ratio is zero in planes z >= Z (the image is zero there): P3 does
    // not write them and this pass reads them as zeros
    ModOTF m4{H2, scale_n};
    m4.zn = id.z;
    CL_TRY(z_pass(ctx, pe, m4, ws.S, ws.S));
    EpiRLProduct epi;
    epi.cur = (k == 0) ? nullptr : ws.u;
    epi.g = u0;
    epi.scale = sk;
    epi.unew = ws.u;
    epi.partial = ws.partial;
    epi.w = wv;
    epi.xmode = P.xmode;
    epi.acc = 0.0;
    epi.nblocks = ws.iscal;  // the partials' count, as launched
    if (k + 1 < iters)
      CL_TRY(xy_inv_fwd(ctx, pe, epi, ws.S));
    else
      CL_TRY(xy_inverse(ctx, pe, epi, ws.S));
    if (rescale) {
      // s = E / sum u' by one block in a fixed order.  A last-block ticket
      // in the product pass itself cost more: each of its blocks then waited
      // for an atomic's round trip before it could exit.
      count_small();
      CLARITY_LAUNCH_PDL(k_finish_rl_scale, 1, kFinishThreads, 0, st, pdl_enabled())(
          ws.partial, ws.iscal, ws.dscal + 0, ws.dscal + 1, sdev);
      CL_CHECK(cudaGetLastError());
    }
  }
  if (idiv && iters > 0) {
    // idiv[iters]: the result's own I-divergence (h * s u', one more forward
    // transform, z pass and xy inverse that only accumulates)
    CL_TRY(xy_forward(ctx, pe, ProWork{ws.u, rescale ? sdev : nullptr, wv, P.xmode}, ws.S));
    CL_TRY(z_pass(ctx, pe, ModOTF{H, scale_n}, ws.S, ws.S));
    MidRLRatio tr{g, P.xmode};
    tr.idiv_partial = ws.partial;
    tr.nblocks = ws.iscal + 1;
    CL_TRY(xy_inverse(ctx, pe, tr, ws.S));
    count_small();
    CLARITY_LAUNCH(k_finish_sum_np, 1, 256, 0, st)(ws.partial, ws.iscal + 1, idiv + iters);
    CL_CHECK(cudaGetLastError());
  }
  return Status::Ok();
}

// The conjugated OTF (ws.HG) from ws.H, for the correlation opt-ins.
static Status conj_otf(Context& ctx, const PlanEntry& pe, Workspace& ws) {
  if (!ws.HG) CL_CHECK(dev_alloc((void**)&ws.HG, sizeof(float2) * (size_t)ws.spec_cap));
  count_small();
  CLARITY_LAUNCH(k_conj_spectrum, kReduceBlocks, 256, 0, ctx.exec_stream())(ws.H, ws.HG,
                                                                            pe.P.spec_elems);
  CL_CHECK(cudaGetLastError());
  return Status::Ok();
}

// One Richardson-Lucy solve on prepared plan and workspace, enqueued on
// ctx.exec_stream(): OTF, the iterations, the clipped result.  correlate:
// the second convolution of each iteration uses the conjugated OTF (a
// correlation with the kernel; the reference convolves twice,
// src/MaximumLikelihoodDeconvolve.cxx:57,65).
static Status rl_solve(Context& ctx, const PlanEntry& pe, Workspace& ws, const float* img,
                       Dims id, const float* ker, Dims kd, Dims wd, float* out, int iters,
                       const float* start = nullptr, double* idiv = nullptr,
                       bool correlate = false) {
  cudaStream_t st = ctx.exec_stream();
  if (iters <= 0) {
    // no iteration: the estimate RL would start from (the reference leaves
    // the output unwritten; here the input image, or `start`)
    const float* est = start ? start : img;
    count_small();
    CLARITY_LAUNCH(k_copy, kReduceBlocks, 256, 0, st)(est, out, id.n());
    CL_CHECK(cudaGetLastError());
    if (idiv) {
      // idiv[0]: that estimate's own I-divergence (one convolution)
      const VolPlan& P = pe.P;
      CL_TRY(make_otf(ctx, pe, ker, kd, wd, ws.H, nullptr));
      CL_TRY(xy_forward(ctx, pe, ProImage{image_src(est, id), P.xmode}, ws.S));
      CL_TRY(z_pass(ctx, pe, ModOTF{ws.H, inv_volume(wd)}, ws.S, ws.S));
      MidRLRatio tr{image_src(img, id), P.xmode};
      tr.idiv_partial = ws.partial;
      tr.nblocks = ws.iscal + 1;
      CL_TRY(xy_inverse(ctx, pe, tr, ws.S));
      count_small();
      CLARITY_LAUNCH(k_finish_sum_np, 1, 256, 0, st)(ws.partial, ws.iscal + 1, idiv);
      CL_CHECK(cudaGetLastError());
    }
    return Status::Ok();
  }
  CL_TRY(make_otf(ctx, pe, ker, kd, wd, ws.H, nullptr));
  RLRoles roles;
  if (correlate) {
    CL_TRY(conj_otf(ctx, pe, ws));
    roles.otf2 = ws.HG;
  }
  CL_TRY(rl_core(ctx, pe, ws, img, id, wd, iters, true, start, idiv, roles));
  count_small();
  CLARITY_LAUNCH(k_clip, kReduceBlocks, 256, 0, st)(ws.u, wd.x, wd.y, out, id.x, id.y, id.z,
                                                    ws.fscal);
  CL_CHECK(cudaGetLastError());
  return Status::Ok();
}

// Runs a scope's enqueues on another stream of the context.
struct StreamScope {
  Context& ctx;
  bool had;
  cudaStream_t saved;
  StreamScope(Context& c, cudaStream_t s)
      : ctx(c), had(c.has_user_stream()), saved(c.exec_stream()) {
    c.set_stream(s);
  }
  ~StreamScope() {
    if (had) ctx.set_stream(saved);
    else ctx.clear_stream();
  }
};

Status run_rl(Context& ctx, const float* img, Dims id, const float* ker,
              Dims kd, float* out, int iters) {
  const PlanEntry* pe;
  Workspace* ws;
  Dims wd;
  CL_TRY(setup(ctx, id, kd, &pe, &ws, &wd));
  return rl_solve(ctx, *pe, *ws, img, id, ker, kd, wd, out, iters);
}

Status run_rl_correlate(Context& ctx, const float* img, Dims id, const float* ker, Dims kd,
                        float* out, int iters) {
  const PlanEntry* pe;
  Workspace* ws;
  Dims wd;
  CL_TRY(setup(ctx, id, kd, &pe, &ws, &wd));
  return rl_solve(ctx, *pe, *ws, img, id, ker, kd, wd, out, iters, nullptr, nullptr, true);
}

Status run_rl_ex(Context& ctx, const float* img, Dims id, const float* ker, Dims kd,
                 const float* start, float* out, int iters, double* idiv) {
  const PlanEntry* pe;
  Workspace* ws;
  Dims wd;
  CL_TRY(setup(ctx, id, kd, &pe, &ws, &wd));
  return rl_solve(ctx, *pe, *ws, img, id, ker, kd, wd, out, iters, start, idiv);
}

// Accelerated Richardson-Lucy (Biggs and Andrews, Applied Optics
// 36(8):1766-1775, 1997; no reference counterpart).  Per iteration:
//   P1 xy forward of y = max(0, x + alpha (x - x_prev)), y stored (ProAccel)
//   P2-P4 as plain RL (z, ratio, z) -- the ratio pass may trace I-div at y
//   P5 xy inverse, u' = y * (h*r), FP64 sums -> s = E / sum u'
//   x_next = s u', g_k = x_next - y, sums of g_k g_{k-1}, g_{k-1}^2 -> alpha
// The three estimate buffers rotate (x_prev, x, x_next); idiv as run_rl_ex,
// its entries k < iters taken at y_k.
Status run_rl_accel(Context& ctx, const float* img, Dims id, const float* ker, Dims kd,
                    const float* start, float* out, int iters, double* idiv) {
  const PlanEntry* pe;
  Workspace* ws;
  Dims wd;
  CL_TRY(setup(ctx, id, kd, &pe, &ws, &wd));
  cudaStream_t st = ctx.exec_stream();
  if (iters <= 0) {
    count_small();
    CLARITY_LAUNCH(k_copy, kReduceBlocks, 256, 0, st)(start ? start : img, out, id.n());
    CL_CHECK(cudaGetLastError());
    return Status::Ok();
  }
  const VolPlan& P = pe->P;
  const long long n = wd.n();
  CL_TRY(ensure_volumes(ws->accel, &ws->accel_cap, n));
  // partials: one per XY block for the flux sum, two per reduce block for
  // the extrapolation sums
  {
    long long pc = ws->partial_cap;
    CL_TRY(ensure(&ws->partial, &pc, 2 * (long long)kReduceBlocks));
    ws->partial_cap = (int)pc;
  }
  CL_TRY(make_otf(ctx, *pe, ker, kd, wd, ws->H, nullptr));
  const ImageSrc g = image_src(img, id);
  const WorkVol wv{wd.x, wd.y, wd.z};
  const float scale_n = inv_volume(wd);
  float* B[3] = {ws->accel[0], ws->accel[1], ws->accel[2]};
  float* Y = ws->accel[3];
  float* G = ws->accel[4];
  float* alpha = ws->fscal + 6;
  float* sdev = ws->fscal;
  int xi = 0, pi = 0, ui = 1;  // x, x_prev, x_next buffers (x_prev = x at first)
  CL_TRY(reduce_sum_into(ctx, img, id.n(), ws->partial, ws->dscal + 0));
  count_small();
  CLARITY_LAUNCH(k_pad_image, kReduceBlocks, 256, 0, st)(start ? image_src(start, id) : g, wv,
                                                         B[0]);
  CL_CHECK(cudaMemsetAsync(alpha, 0, sizeof(float), st));
  for (int k = 0; k < iters; ++k) {
    CL_TRY(xy_forward(ctx, *pe, ProAccel{B[xi], B[pi], alpha, Y, wv, P.xmode}, ws->S));
    ModOTF m2{ws->H, scale_n};
    m2.zout = id.z;  // the ratio pass reads planes z < Z only
    CL_TRY(z_pass(ctx, *pe, m2, ws->S, ws->S));
    MidRLRatio ratio{g, P.xmode};
    if (idiv) {
      ratio.idiv_partial = ws->partial;
      ratio.nblocks = ws->iscal + 1;
    }
    CL_TRY(xy_inv_fwd(ctx, *pe, ratio, ws->S));
    if (idiv) {
      count_small();
      CLARITY_LAUNCH(k_finish_sum_np, 1, 256, 0, st)(ws->partial, ws->iscal + 1, idiv + k);
      CL_CHECK(cudaGetLastError());
    }
    ModOTF m4{ws->H, scale_n};
    m4.zn = id.z;
    CL_TRY(z_pass(ctx, *pe, m4, ws->S, ws->S));
    EpiRLProduct epi;
    epi.cur = Y;
    epi.g = g;
    epi.scale = nullptr;
    epi.unew = B[ui];
    epi.partial = ws->partial;
    epi.w = wv;
    epi.xmode = P.xmode;
    epi.acc = 0.0;
    epi.nblocks = ws->iscal;
    CL_TRY(xy_inverse(ctx, *pe, epi, ws->S));
    count_small();
    CLARITY_LAUNCH_PDL(k_finish_rl_scale, 1, kFinishThreads, 0, st, pdl_enabled())(
        ws->partial, ws->iscal, ws->dscal + 0, ws->dscal + 1, sdev);
    count_small();
    CLARITY_LAUNCH(k_accel_update, kReduceBlocks, 256, 0, st)(B[ui], Y, G, sdev, k == 0 ? 1 : 0,
                                                              n, ws->partial);
    CL_CHECK(cudaGetLastError());
    if (k > 0) {
      count_small();
      CLARITY_LAUNCH(k_finish_alpha, 1, 256, 0, st)(ws->partial, kReduceBlocks, alpha);
      CL_CHECK(cudaGetLastError());
    }
    // rotate: x_prev <- x, x <- x_next, x_next <- the free buffer
    pi = xi;
    xi = ui;
    ui = 3 - pi - xi;
  }
  if (idiv) {
    CL_TRY(xy_forward(ctx, *pe, ProWork{B[xi], nullptr, wv, P.xmode}, ws->S));
    CL_TRY(z_pass(ctx, *pe, ModOTF{ws->H, scale_n}, ws->S, ws->S));
    MidRLRatio tr{g, P.xmode};
    tr.idiv_partial = ws->partial;
    tr.nblocks = ws->iscal + 1;
    CL_TRY(xy_inverse(ctx, *pe, tr, ws->S));
    count_small();
    CLARITY_LAUNCH(k_finish_sum_np, 1, 256, 0, st)(ws->partial, ws->iscal + 1, idiv + iters);
    CL_CHECK(cudaGetLastError());
  }
  count_small();
  CLARITY_LAUNCH(k_clip, kReduceBlocks, 256, 0, st)(B[xi], wd.x, wd.y, out, id.x, id.y, id.z,
                                                    nullptr);
  CL_CHECK(cudaGetLastError());
  return Status::Ok();
}

// Batched Richardson-Lucy.  Set-up (plans, possibly autotuned, and one
// workspace per volume) happens first, outside any capture; then every
// volume's solve is issued on batch stream i % nstreams, forked from and
// joined back to the caller's stream by events, either directly or captured
// into one CUDA graph that later calls with the same volumes replay.
// RL set-up of one volume before its first iteration (as rl_solve and
// rl_core): OTF, energy E = sum of the image, first forward transform.
static Status rl_prologue(Context& ctx, const PlanEntry& pe, Workspace& ws, const float* img,
                          Dims id, const float* ker, Dims kd, Dims wd) {
  CL_TRY(make_otf(ctx, pe, ker, kd, wd, ws.H, nullptr));
  CL_TRY(reduce_sum_into(ctx, img, id.n(), ws.partial, ws.dscal + 0));
  return xy_forward(ctx, pe, ProImage{image_src(img, id), pe.P.xmode}, ws.S);
}

Status run_rl_batch(Context& ctx, int n, const float* const* imgs, const Dims* ids,
                    const float* const* kers, const Dims* kds, float* const* outs, int iters,
                    bool use_graph, bool persistent) {
  if (n <= 0) return Status::Ok();
  if (iters <= 0) persistent = false;  // nothing to iterate: the copy of rl_solve
#ifdef CLARITY_HOST_EMULATION
  use_graph = false;  // the emulation runs kernels as they are issued
#endif
  constexpr int kBatchStreams = 8;
  const int ns = std::min(n, kBatchStreams);
  std::vector<const PlanEntry*> pes(n);
  std::vector<Workspace*> wss(n);
  std::vector<Dims> wds(n);
  std::vector<cudaStream_t> bs(ns);
  for (int i = 0; i < n; ++i) {
    if (!imgs[i] || !kers[i] || !outs[i]) {
      Status s;
      s.code = CLARITY_INVALID_ARGUMENT;
      s.msg = "batch volume " + std::to_string(i) + ": NULL pointer";
      return s;
    }
    wds[i] = work_dims(ids[i], kds[i]);
    CL_TRY(ctx.plan(wds[i], &pes[i]));
    CL_TRY(ctx.workspace_slot(i, *pes[i], ids[i], kds[i], &wss[i]));
  }
  for (int j = 0; j < ns; ++j) CL_TRY(ctx.batch_stream(j, &bs[j]));
  void* qbuf = nullptr;
  if (persistent) CL_TRY(ctx.batch_scratch(batch_queue_bytes(n, iters), &qbuf));
  // the caller's stream; a graph is captured on and launched from the
  // context's own stream (capture is not allowed on the legacy default
  // stream), ordered after and before the caller's work by events
  const cudaStream_t caller = ctx.exec_stream();
  const cudaStream_t origin = use_graph ? ctx.own_stream() : caller;
  std::vector<unsigned long long> key;
  key.push_back((unsigned long long)n);
  key.push_back((unsigned long long)iters);
  key.push_back(persistent ? 1ull : 0ull);
  key.push_back((unsigned long long)(uintptr_t)qbuf);
  for (int i = 0; i < n; ++i) {
    for (const void* p : {(const void*)imgs[i], (const void*)kers[i], (const void*)outs[i],
                          (const void*)wss[i]->S, (const void*)wss[i]->H,
                          (const void*)wss[i]->u, (const void*)pes[i]})
      key.push_back((unsigned long long)(uintptr_t)p);
    key.push_back(((unsigned long long)ids[i].x << 42) | ((unsigned long long)ids[i].y << 21) |
                  (unsigned long long)ids[i].z);
    key.push_back(((unsigned long long)kds[i].x << 42) | ((unsigned long long)kds[i].y << 21) |
                  (unsigned long long)kds[i].z);
  }
  // caller -> origin -> caller ordering around a graph launch
  auto after_caller = [&]() -> Status {
    cudaEvent_t e = nullptr;
    CL_CHECK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    cudaError_t r = cudaEventRecord(e, caller);
    if (r == cudaSuccess) r = cudaStreamWaitEvent(origin, e, 0);
    cudaEventDestroy(e);
    CL_CHECK(r);
    return Status::Ok();
  };
  auto before_caller = [&]() -> Status {
    cudaEvent_t e = nullptr;
    CL_CHECK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    cudaError_t r = cudaEventRecord(e, origin);
    if (r == cudaSuccess) r = cudaStreamWaitEvent(caller, e, 0);
    cudaEventDestroy(e);
    CL_CHECK(r);
    return Status::Ok();
  };
  if (use_graph) {
    if (cudaGraphExec_t g = ctx.find_graph(key)) {
      CL_TRY(after_caller());
      CL_CHECK(cudaGraphLaunch(g, origin));
      return before_caller();
    }
  }
  auto issue = [&]() -> Status {
    cudaEvent_t fork = nullptr;
    std::vector<cudaEvent_t> join(ns, nullptr);
    Status st = Status::Ok();
    auto body = [&]() -> Status {
      CL_CHECK(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
      for (int j = 0; j < ns; ++j)
        CL_CHECK(cudaEventCreateWithFlags(&join[j], cudaEventDisableTiming));
      CL_CHECK(cudaEventRecord(fork, origin));
      for (int j = 0; j < ns; ++j) CL_CHECK(cudaStreamWaitEvent(bs[j], fork, 0));
      for (int i = 0; i < n; ++i) {
        StreamScope scope(ctx, bs[i % ns]);
        if (persistent)
          CL_TRY(rl_prologue(ctx, *pes[i], *wss[i], imgs[i], ids[i], kers[i], kds[i], wds[i]));
        else
          CL_TRY(rl_solve(ctx, *pes[i], *wss[i], imgs[i], ids[i], kers[i], kds[i], wds[i],
                          outs[i], iters));
      }
      for (int j = 0; j < ns; ++j) {
        CL_CHECK(cudaEventRecord(join[j], bs[j]));
        CL_CHECK(cudaStreamWaitEvent(origin, join[j], 0));
      }
      if (persistent) {
        // every volume's iterations in one launch, then the clipped results
        CL_TRY(launch_rl_batch(ctx, n, pes.data(), wss.data(), imgs, ids, wds.data(), iters,
                               qbuf, origin));
        for (int i = 0; i < n; ++i) {
          count_small();
          CLARITY_LAUNCH(k_clip, kReduceBlocks, 256, 0, origin)(
              wss[i]->u, wds[i].x, wds[i].y, outs[i], ids[i].x, ids[i].y, ids[i].z,
              wss[i]->fscal);
          CL_CHECK(cudaGetLastError());
        }
      }
      return Status::Ok();
    };
    st = body();
    if (fork) cudaEventDestroy(fork);
    for (cudaEvent_t e : join)
      if (e) cudaEventDestroy(e);
    return st;
  };
  if (!use_graph) return issue();
#ifndef CLARITY_HOST_EMULATION
  CL_CHECK(cudaStreamBeginCapture(origin, cudaStreamCaptureModeThreadLocal));
  set_capturing(true);
  Status st = issue();
  set_capturing(false);
  cudaGraph_t graph = nullptr;
  const cudaError_t ce = cudaStreamEndCapture(origin, &graph);
  if (!st.ok()) {
    if (graph) cudaGraphDestroy(graph);
    return st;
  }
  CL_CHECK(ce);
  cudaGraphExec_t exec = nullptr;
  const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
  cudaGraphDestroy(graph);
  CL_CHECK(ie);
  ctx.add_graph(std::move(key), exec);
  CL_TRY(after_caller());
  CL_CHECK(cudaGraphLaunch(exec, origin));
  CL_TRY(before_caller());
#endif
  return Status::Ok();
}

Status run_blind(Context& ctx, const float* img, Dims id, const float* ker,
                 Dims kd, float* out, int iters) {
  const PlanEntry* pe;
  Workspace* ws;
  Dims wd;
  CL_TRY(setup(ctx, id, kd, &pe, &ws, &wd));
  cudaStream_t st = ctx.exec_stream();
  if (iters <= 0) {
    count_small();
    CLARITY_LAUNCH(k_copy, kReduceBlocks, 256, 0, st)(img, out, id.n());
    CL_CHECK(cudaGetLastError());
    return Status::Ok();
  }
  // h <- h / sum(h) (src/BlindMaximumLikelihoodDeconvolve.cxx:59)
  count_small();
  CLARITY_LAUNCH(k_reduce_sum, kReduceBlocks, 256, 0, st)(ker, kd.n(), ws->partial);
  count_small();
  CLARITY_LAUNCH(k_finish_inverse, 1, 256, 0, st)(ws->partial, kReduceBlocks, ws->fscal + 2);
  CL_CHECK(cudaGetLastError());
  CL_TRY(make_otf(ctx, *pe, ker, kd, wd, ws->H, ws->fscal + 2));
  CL_TRY(rl_core(ctx, *pe, *ws, img, id, wd, iters, false));
  count_small();
  CLARITY_LAUNCH(k_clip, kReduceBlocks, 256, 0, st)(ws->u, wd.x, wd.y, out, id.x, id.y, id.z,
                                        nullptr);
  CL_CHECK(cudaGetLastError());
  return Status::Ok();
}

// Jansen-van Cittert: the first update reads the padded image; every update
// is a z pass (h * i) plus one fused XY pass (inverse, JVC update, store i',
// forward transform of i' for the next update).
// Blind ML with the PSF update the reference leaves disabled
// (src/BlindMaximumLikelihoodDeconvolve.cxx:50-99, the commented-out :96):
// alternating updates -- per outer iteration one object step
// o <- o (h * (g / (h * o))) with the current PSF, then psf_subiters PSF steps
// h <- h (o * (g / (h * o))) renormalised to unit sum (:59) with the new
// object.  Each step is one RL iteration of rl_core with the roles set: the
// PSF step deconvolves by the object (its spectrum as the OTF) and rescales
// to 1.  The object and PSF estimates live on the work box; psf_out (optional)
// receives the PSF on the kernel's grid.
// ------------------------------------------------- I-divergence restoration
// Markham and Conchello (J. Opt. Soc. Am. A 18(5), 2001), the method the
// reference declares (Clarity.h.in:294-319) and leaves a stub
// (src/IDivergenceDeconvolve.cxx).  Minimises sum g ln(g/gh) + gh - g +
// alpha sum s^2 over the work box (g zero-padded, gh = h * s) with s = a^2,
// by Polak-Ribiere conjugate gradients on a; the step solves dJ/dl = 0 by
// kIdivNewton Newton steps on the exact quadratic gh(l) = gh + l h*(2ad) +
// l^2 h*(dd).  Per-voxel line-search terms and all sums in FP64.
static constexpr int kIdivNewton = 4;

__device__ __forceinline__ double idiv_ratio(double g, double b) { return b > 1e-5 ? g / b : 0.0; }

// a = sqrt(g) on the work box (g zero-padded)
__global__ void k_idiv_start(ImageSrc g, WorkVol w, float* __restrict__ a) {
  const long long n = (long long)w.nx * w.ny * w.nz;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % w.nx);
    const long long r = i / w.nx;
    const float v = g.at(x, (int)(r % w.ny), (int)(r / w.ny));
    a[i] = sqrtf(v > 0.f ? v : 0.f);
  }
}

// t = c * a * b (b == nullptr: c * a * a)
__global__ void k_idiv_prod(const float* __restrict__ a, const float* __restrict__ b, float c,
                            float* __restrict__ t, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const float bv = b ? b[i] : a[i];
    t[i] = c == 1.f ? a[i] * bv : c * a[i] * bv;
  }
}

// t = 1 - g / gh (the ratio 0 where gh <= 1e-5)
__global__ void k_idiv_resid(ImageSrc g, WorkVol w, const float* __restrict__ gh,
                             float* __restrict__ t) {
  const long long n = (long long)w.nx * w.ny * w.nz;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % w.nx);
    const long long r = i / w.nx;
    const float gv = g.at(x, (int)(r % w.ny), (int)(r / w.ny));
    t[i] = (float)(1.0 - idiv_ratio(gv, gh[i]));
  }
}

// grn = 2 a (q + 2 alpha a^2)
__global__ void k_idiv_grad(const float* __restrict__ a, const float* __restrict__ q, float alpha2,
                            float* __restrict__ grn, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const float av = a[i];
    grn[i] = 2.f * av * (q[i] + alpha2 * av * av);
  }
}

// d = -gr (first direction)
__global__ void k_idiv_negate(const float* __restrict__ gr, float* __restrict__ d, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    d[i] = -gr[i];
}

// FP64 sums of dJ/dl and d2J/dl2 at l = *lam (partial[b], partial[nb + b])
__global__ void k_idiv_newton_sums(ImageSrc g, WorkVol w, const float* __restrict__ gh,
                                   const float* __restrict__ p1, const float* __restrict__ p2,
                                   const float* __restrict__ a, const float* __restrict__ d,
                                   const double* __restrict__ lam, double alpha,
                                   double* __restrict__ partial) {
  const long long n = (long long)w.nx * w.ny * w.nz;
  const double l = *lam;
  double f1 = 0, f2 = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % w.nx);
    const long long r = i / w.nx;
    const double gv = g.at(x, (int)(r % w.ny), (int)(r / w.ny));
    const double q2 = p2[i];
    const double ghl = (double)gh[i] + l * (double)p1[i] + l * l * q2;
    const double gp = (double)p1[i] + 2.0 * l * q2;
    const double rr = idiv_ratio(gv, ghl);
    f1 += (1.0 - rr) * gp;
    f2 += (ghl > 1e-5 ? rr / ghl : 0.0) * gp * gp + (1.0 - rr) * 2.0 * q2;
    const double dd = d[i], sl = (double)a[i] + l * dd;
    f1 += 4.0 * alpha * sl * sl * sl * dd;
    f2 += 12.0 * alpha * sl * sl * dd * dd;
  }
  block_sum_store(f1, partial + 0 * gridDim.x);
  block_sum_store(f2, partial + 1 * gridDim.x);
}

// one Newton step: l <- max(0, l - f1/f2) when f2 > 0
__global__ void k_idiv_newton_finish(const double* partial, int np, double* lam) {
  const double f1 = block_total(partial, np);
  __syncthreads();
  const double f2 = block_total(partial + np, np);
  if (threadIdx.x == 0 && f2 > 0) {
    double l = *lam - f1 / f2;
    *lam = l < 0 ? 0 : l;
  }
}

// a += l d, gh += l p1 + l^2 p2
__global__ void k_idiv_move(float* __restrict__ a, const float* __restrict__ d,
                            float* __restrict__ gh, const float* __restrict__ p1,
                            const float* __restrict__ p2, const double* __restrict__ lam,
                            long long n) {
  const double l = *lam;
  const float lf = (float)l, l2 = (float)(l * l);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    a[i] = a[i] + lf * d[i];
    gh[i] = gh[i] + lf * p1[i] + l2 * p2[i];
  }
}

// Polak-Ribiere sums: grn . (grn - gr) and gr . gr
__global__ void k_idiv_pr_sums(const float* __restrict__ grn, const float* __restrict__ gr,
                               long long n, double* __restrict__ partial) {
  double s1 = 0, s2 = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const double a = grn[i], b = gr[i];
    s1 += a * (a - b);
    s2 += b * b;
  }
  block_sum_store(s1, partial + 0 * gridDim.x);
  block_sum_store(s2, partial + 1 * gridDim.x);
}

// beta = max(0, s1 / s2); d = -grn + beta d; gr = grn.  The sums are
// finished by every block (fixed order, identical results), so one launch
// both finishes and applies them.
__global__ void k_idiv_direction(const double* partial, int np, float* __restrict__ d,
                                 const float* __restrict__ grn, float* __restrict__ gr,
                                 long long n) {
  __shared__ float sbeta;
  const double s1 = block_total(partial, np);
  __syncthreads();
  const double s2 = block_total(partial + np, np);
  if (threadIdx.x == 0) {
    double b = s2 > 0 ? s1 / s2 : 0.0;
    sbeta = (float)(b < 0 ? 0 : b);
  }
  __syncthreads();
  const float beta = sbeta;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const float gn = grn[i];
    d[i] = -gn + beta * d[i];
    gr[i] = gn;
  }
}

// v <- h (x) v on the work box (in place): forward transform, the spectral
// product with `otf` (H for a convolution, conj(H) for a correlation) and 1/N,
// inverse transform.
static Status conv_work(Context& ctx, const PlanEntry& pe, Workspace& ws, const float2* otf,
                        float* v, Dims wd) {
  const VolPlan& P = pe.P;
  const WorkVol wv{wd.x, wd.y, wd.z};
  CL_TRY(xy_forward(ctx, pe, ProWork{v, nullptr, wv, P.xmode}, ws.S));
  CL_TRY(z_pass(ctx, pe, ModOTF{otf, inv_volume(wd)}, ws.S, ws.S));
  CL_TRY(xy_inverse(ctx, pe, EpiWork{v, wv, P.xmode}, ws.S));
  return Status::Ok();
}

Status run_idiv_cg(Context& ctx, const float* img, Dims id, const float* ker, Dims kd,
                   float* out, int iters, float alpha) {
  const PlanEntry* pe;
  Workspace* ws;
  Dims wd;
  CL_TRY(setup(ctx, id, kd, &pe, &ws, &wd));
  cudaStream_t st = ctx.exec_stream();
  const long long n = wd.n();
  CL_TRY(ensure_volumes(ws->accel, &ws->accel_cap, n));
  CL_TRY(ensure_volumes(ws->xbuf, &ws->xbuf_cap, n));
  {
    long long pc = ws->partial_cap;
    CL_TRY(ensure(&ws->partial, &pc, 2 * (long long)kReduceBlocks));
    ws->partial_cap = (int)pc;
  }
  if (!ws->HG) CL_CHECK(dev_alloc((void**)&ws->HG, sizeof(float2) * (size_t)ws->spec_cap));
  CL_TRY(make_otf(ctx, *pe, ker, kd, wd, ws->H, nullptr));
  count_small();
  CLARITY_LAUNCH(k_conj_spectrum, kReduceBlocks, 256, 0, st)(ws->H, ws->HG, pe->P.spec_elems);
  CL_CHECK(cudaGetLastError());
  const ImageSrc g = image_src(img, id);
  const WorkVol wv{wd.x, wd.y, wd.z};
  float* a = ws->accel[0];
  float* d = ws->accel[1];
  float* gr = ws->accel[2];
  float* grn = ws->accel[3];
  float* gh = ws->accel[4];
  float* p1 = ws->xbuf[0];
  float* p2 = ws->xbuf[1];
  float* t = ws->u;
  double* lam = ws->dscal + 4;
  const float alpha2 = 2.f * alpha;
  auto gradient = [&]() -> Status {
    count_small();
    CLARITY_LAUNCH(k_idiv_resid, kReduceBlocks, 256, 0, st)(g, wv, gh, t);
    CL_CHECK(cudaGetLastError());
    CL_TRY(conv_work(ctx, *pe, *ws, ws->HG, t, wd));
    count_small();
    CLARITY_LAUNCH(k_idiv_grad, kReduceBlocks, 256, 0, st)(a, t, alpha2, grn, n);
    CL_CHECK(cudaGetLastError());
    return Status::Ok();
  };
  count_small();
  CLARITY_LAUNCH(k_idiv_start, kReduceBlocks, 256, 0, st)(g, wv, a);
  count_small();
  CLARITY_LAUNCH(k_idiv_prod, kReduceBlocks, 256, 0, st)(a, nullptr, 1.f, gh, n);
  CL_CHECK(cudaGetLastError());
  CL_TRY(conv_work(ctx, *pe, *ws, ws->H, gh, wd));
  CL_TRY(gradient());
  CL_CHECK(cudaMemcpyAsync(gr, grn, sizeof(float) * (size_t)n, cudaMemcpyDeviceToDevice, st));
  count_small();
  CLARITY_LAUNCH(k_idiv_negate, kReduceBlocks, 256, 0, st)(grn, d, n);
  CL_CHECK(cudaGetLastError());
  for (int k = 0; k < iters; ++k) {
    count_small();
    CLARITY_LAUNCH(k_idiv_prod, kReduceBlocks, 256, 0, st)(a, d, 2.f, p1, n);
    CL_CHECK(cudaGetLastError());
    CL_TRY(conv_work(ctx, *pe, *ws, ws->H, p1, wd));
    count_small();
    CLARITY_LAUNCH(k_idiv_prod, kReduceBlocks, 256, 0, st)(d, nullptr, 1.f, p2, n);
    CL_CHECK(cudaGetLastError());
    CL_TRY(conv_work(ctx, *pe, *ws, ws->H, p2, wd));
    CL_CHECK(cudaMemsetAsync(lam, 0, sizeof(double), st));
    for (int m = 0; m < kIdivNewton; ++m) {
      count_small();
      CLARITY_LAUNCH(k_idiv_newton_sums, kReduceBlocks, 256, 0, st)(g, wv, gh, p1, p2, a, d, lam,
                                                                    (double)alpha, ws->partial);
      count_small();
      CLARITY_LAUNCH(k_idiv_newton_finish, 1, 256, 0, st)(ws->partial, kReduceBlocks, lam);
      CL_CHECK(cudaGetLastError());
    }
    count_small();
    CLARITY_LAUNCH(k_idiv_move, kReduceBlocks, 256, 0, st)(a, d, gh, p1, p2, lam, n);
    CL_CHECK(cudaGetLastError());
    CL_TRY(gradient());
    count_small();
    CLARITY_LAUNCH(k_idiv_pr_sums, kReduceBlocks, 256, 0, st)(grn, gr, n, ws->partial);
    count_small();
    CLARITY_LAUNCH(k_idiv_direction, kReduceBlocks, 256, 0, st)(ws->partial, kReduceBlocks, d, grn,
                                                                gr, n);
    CL_CHECK(cudaGetLastError());
  }
  count_small();
  CLARITY_LAUNCH(k_idiv_prod, kReduceBlocks, 256, 0, st)(a, nullptr, 1.f, t, n);
  count_small();
  CLARITY_LAUNCH(k_clip, kReduceBlocks, 256, 0, st)(t, wd.x, wd.y, out, id.x, id.y, id.z, nullptr);
  CL_CHECK(cudaGetLastError());
  return Status::Ok();
}

Status run_blind_psf(Context& ctx, const float* img, Dims id, const float* ker, Dims kd,
                     float* out, float* psf_out, int iters, int psf_subiters) {
  const PlanEntry* pe;
  Workspace* ws;
  Dims wd;
  CL_TRY(setup(ctx, id, kd, &pe, &ws, &wd));
  cudaStream_t st = ctx.exec_stream();
  const VolPlan& P = pe->P;
  const long long n = wd.n();
  CL_TRY(ensure_volumes(ws->accel, &ws->accel_cap, n));
  if (!ws->HG) CL_CHECK(dev_alloc((void**)&ws->HG, sizeof(float2) * (size_t)ws->spec_cap));
  float* o = ws->accel[0];
  float* h = ws->accel[1];
  const WorkVol wv{wd.x, wd.y, wd.z};
  // h = pad/shift(kernel) / sum(kernel); o = the image on the work box
  count_small();
  CLARITY_LAUNCH(k_reduce_sum, kReduceBlocks, 256, 0, st)(ker, kd.n(), ws->partial);
  count_small();
  CLARITY_LAUNCH(k_finish_inverse, 1, 256, 0, st)(ws->partial, kReduceBlocks, ws->fscal + 2);
  count_small();
  CLARITY_LAUNCH(k_pad_scaled, kReduceBlocks, 256, 0, st)(
      padded(ker, kd, wd, -kd.x / 2, -kd.y / 2, -kd.z / 2), ws->fscal + 2, h);
  count_small();
  CLARITY_LAUNCH(k_pad_image, kReduceBlocks, 256, 0, st)(image_src(img, id), wv, o);
  CL_CHECK(cudaGetLastError());
  RLRoles obj;
  obj.otf = ws->H;
  obj.start_dims = wd;
  RLRoles psf;
  psf.otf = ws->HG;
  psf.start_dims = wd;
  psf.unit_energy = true;
  for (int k = 0; k < iters; ++k) {
    CL_TRY(xy_forward(ctx, *pe, ProWork{h, nullptr, wv, P.xmode}, ws->H));
    CL_TRY(z_pass(ctx, *pe, ModForward{}, ws->H, ws->H));
    CL_TRY(rl_core(ctx, *pe, *ws, img, id, wd, 1, false, o, nullptr, obj));
    CL_CHECK(cudaMemcpyAsync(o, ws->u, sizeof(float) * (size_t)n, cudaMemcpyDeviceToDevice, st));
    if (psf_subiters > 0) {
      CL_TRY(xy_forward(ctx, *pe, ProWork{o, nullptr, wv, P.xmode}, ws->HG));
      CL_TRY(z_pass(ctx, *pe, ModForward{}, ws->HG, ws->HG));
    }
    for (int j = 0; j < psf_subiters; ++j) {
      CL_TRY(rl_core(ctx, *pe, *ws, img, id, wd, 1, true, h, nullptr, psf));
      count_small();
      CLARITY_LAUNCH(k_scale_copy, kReduceBlocks, 256, 0, st)(ws->u, ws->fscal, h, n);
      CL_CHECK(cudaGetLastError());
    }
  }
  count_small();
  CLARITY_LAUNCH(k_clip, kReduceBlocks, 256, 0, st)(o, wd.x, wd.y, out, id.x, id.y, id.z, nullptr);
  if (psf_out) {
    count_small();
    CLARITY_LAUNCH(k_unpad_psf, kReduceBlocks, 256, 0, st)(h, wd, kd, psf_out);
  }
  CL_CHECK(cudaGetLastError());
  return Status::Ok();
}

// Sampled Gaussian smoothing kernel of the work-box size (smoothed JVC):
// exp(-d^2 / (2 sigma^2)) per axis about the centre n/2, a delta along an
// axis with sigma <= 0, normalised to unit sum in double and rounded to float.
// Treated as a PSF (pad/shift by -n/2), its OTF convolves the estimate with a
// Gaussian centred at the origin.
static std::vector<float> gauss_kernel(Dims wd, const float* sigma) {
  const int n[3] = {wd.x, wd.y, wd.z};
  std::vector<double> ax[3];
  for (int d = 0; d < 3; ++d) {
    ax[d].resize(n[d]);
    const int c = n[d] / 2;
    const double s = sigma[d];
    for (int i = 0; i < n[d]; ++i) {
      const double t = i - c;
      ax[d][i] = s > 0 ? std::exp(-t * t / (2.0 * s * s)) : (i == c ? 1.0 : 0.0);
    }
  }
  double sum = 0;
  for (int z = 0; z < n[2]; ++z)
    for (int y = 0; y < n[1]; ++y)
      for (int x = 0; x < n[0]; ++x) sum += ax[2][z] * ax[1][y] * ax[0][x];
  std::vector<float> k((size_t)wd.n());
  size_t o = 0;
  for (int z = 0; z < n[2]; ++z)
    for (int y = 0; y < n[1]; ++y)
      for (int x = 0; x < n[0]; ++x) k[o++] = (float)(ax[2][z] * ax[1][y] * ax[0][x] / sum);
  return k;
}

// JVC (src/JansenVanCittertDeconvolve.cxx:311-389), two fused passes per
// update.  Smoothed JVC (smooth_interval > 0; the reference body writes
// zeros, src/SmoothedJansenVanCittertDeconvolve.cxx:27-40): after every
// smooth_interval-th update the work-box estimate is convolved with
// gauss_kernel(smooth_sigma) -- one z pass with the kernel's OTF and one xy
// pass that stores the smoothed estimate (and transforms it on).
Status run_jvc(Context& ctx, const float* img, Dims id, const float* ker,
               Dims kd, float* out, int iters, float /*image_max*/,
               const float* smooth_sigma, int smooth_interval) {
  const PlanEntry* pe;
  Workspace* ws;
  Dims wd;
  CL_TRY(setup(ctx, id, kd, &pe, &ws, &wd));
  const VolPlan& P = pe->P;
  cudaStream_t st = ctx.exec_stream();
  // A = max(unpadded image) / 2 (src/JansenVanCittertDeconvolve.cxx:324)
  float* pmax = reinterpret_cast<float*>(ws->partial);
  count_small();
  CLARITY_LAUNCH(k_reduce_max, kReduceBlocks, 256, 0, st)(img, id.n(), pmax);
  count_small();
  CLARITY_LAUNCH(k_finish_jvc, 1, 32, 0, st)(pmax, kReduceBlocks, ws->fscal + 4);
  CL_CHECK(cudaGetLastError());
  // A and invASq are needed as kernel arguments: read them back once.
  float hc[2];
  CL_CHECK(cudaMemcpyAsync(hc, ws->fscal + 4, sizeof(hc), cudaMemcpyDeviceToHost, st));
  CL_CHECK(cudaStreamSynchronize(st));
  CL_TRY(make_otf(ctx, *pe, ker, kd, wd, ws->H, nullptr));
  const bool smooth = smooth_sigma != nullptr && smooth_interval > 0;
  if (smooth) {
    // the smoothing kernel's OTF; ws->u holds the kernel meanwhile (the
    // estimate is first written by the first update)
    if (!ws->HG) CL_CHECK(dev_alloc((void**)&ws->HG, sizeof(float2) * (size_t)ws->spec_cap));
    const std::vector<float> gk = gauss_kernel(wd, smooth_sigma);
    CL_CHECK(cudaMemcpyAsync(ws->u, gk.data(), sizeof(float) * gk.size(),
                             cudaMemcpyHostToDevice, st));
    CL_TRY(make_otf(ctx, *pe, ws->u, wd, wd, ws->HG, nullptr));
    CL_CHECK(cudaStreamSynchronize(st));  // gk is pageable host memory
  }
  const ImageSrc g = image_src(img, id);
  const WorkVol wv{wd.x, wd.y, wd.z};
  const float scale_n = inv_volume(wd);
  const int total = iters > 1 ? iters : 1;
  CL_TRY(xy_forward(ctx, *pe, ProImage{g, P.xmode}, ws->S));
  for (int k = 0; k < total; ++k) {
    const bool last = k + 1 == total;
    const bool smooth_now = smooth && (k + 1) % smooth_interval == 0;
    CL_TRY(z_pass(ctx, *pe, ModOTF{ws->H, scale_n}, ws->S, ws->S));
    EpiJVC epi{k == 0 ? nullptr : ws->u, g, ws->u, hc[0], hc[1], wv, P.xmode};
    if (!last || smooth_now)
      CL_TRY(xy_inv_fwd(ctx, *pe, epi, ws->S));
    else
      CL_TRY(xy_inverse(ctx, *pe, epi, ws->S));
    if (smooth_now) {
      CL_TRY(z_pass(ctx, *pe, ModOTF{ws->HG, scale_n}, ws->S, ws->S));
      const EpiWork ew{ws->u, wv, P.xmode};
      if (!last)
        CL_TRY(xy_inv_fwd(ctx, *pe, ew, ws->S));
      else
        CL_TRY(xy_inverse(ctx, *pe, ew, ws->S));
    }
  }
  count_small();
  CLARITY_LAUNCH(k_clip, kReduceBlocks, 256, 0, st)(ws->u, wd.x, wd.y, out, id.x, id.y, id.z,
                                        nullptr);
  CL_CHECK(cudaGetLastError());
  return Status::Ok();
}

Status run_idivergence(Context& ctx, const float* g, const float* ghat,
                       long long n, double* result) {
  cudaStream_t st = ctx.exec_stream();
  double* part = nullptr;
  double* d = nullptr;
  CL_CHECK(dev_alloc((void**)&part, sizeof(double) * kReduceBlocks));
  CL_CHECK(dev_alloc((void**)&d, sizeof(double)));
  count_small();
  CLARITY_LAUNCH(k_idiv, kReduceBlocks, 256, 0, st)(g, ghat, n, part);
  count_small();
  CLARITY_LAUNCH(k_finish_sum, 1, 256, 0, st)(part, kReduceBlocks, d);
  cudaError_t e = cudaMemcpyAsync(result, d, sizeof(double), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaFree(part);
  cudaFree(d);
  CL_CHECK(e);
  return Status::Ok();
}

}  // namespace clarity
