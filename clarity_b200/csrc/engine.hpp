// engine.hpp -- internal C++ interface between the C ABI layer and the CUDA
// engine.  Everything here works on DEVICE pointers and enqueues on the
// context stream; the C ABI layer owns host<->device staging.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/clarity.h"
#include "plan.hpp"

namespace clarity {

struct Dims {
  int x, y, z;
  long long n() const { return (long long)x * y * z; }
};

// Error with a ClarityResult_t code and a message for clarityx_last_error.
struct Status {
  ClarityResult_t code = CLARITY_SUCCESS;
  std::string msg;
  bool ok() const { return code == CLARITY_SUCCESS; }
  static Status Ok() { return Status(); }
};

Status status_from_cuda(cudaError_t e, const char* what);

// Plans are built once per work box and cached; tables live on the device.
struct PlanEntry {
  VolPlan P;
  float2* tw = nullptr;  // twiddle tables (FP64-generated, rounded)
  int* xrev = nullptr;   // natural x frequency -> smem slot after x passes
  int* err = nullptr;    // the context's error word (device alias; not owned)
};


// Device allocation that honours the host-side fault injector.
cudaError_t dev_alloc(void** p, size_t bytes);
void set_alloc_failure_countdown(int n);

// Reusable device buffers for one work box.
struct Workspace {
  float2* S = nullptr;     // work spectrum (S layout)
  float2* H = nullptr;     // OTF (S layout)
  float2* HG = nullptr;    // smoothing-kernel OTF (S layout; smoothed JVC only)
  float* u = nullptr;      // work-box real volume (estimate)
  float* img = nullptr;    // unpadded image
  float* ker = nullptr;    // unpadded kernel
  double* partial = nullptr;
  double* dscal = nullptr; // [0] energy, [1] last sum, [2..] misc
  float* fscal = nullptr;  // [0] deferred scale, [1] ones, [2..] misc
  int* iscal = nullptr;    // [0] number of partial sums the last product pass wrote
  float* accel[5] = {};    // accelerated RL: three estimates, extrapolated point, step
  long long accel_cap = 0;
  float* xbuf[2] = {};     // I-divergence restoration: two more work-box volumes
  long long xbuf_cap = 0;
  size_t img_cap = 0, ker_cap = 0;
  long long spec_cap = 0, work_cap = 0;
  int partial_cap = 0;
};

class Context {
 public:
  explicit Context(int device);
  ~Context();
  // Creates the stream and the error word; call once after construction.
  Status init();
  int device() const { return device_; }
  // Error word the kernels write when a bounded wait gives up or a copy
  // address is misaligned: one int of mapped pinned host memory, so the host
  // reads it without a device synchronisation.  Device alias for kernels.
  int* err_dev() const { return err_dev_; }
  cudaStream_t stream() const { return stream_; }
  // The stream work is enqueued on: the caller's (any handle, 0 included,
  // which is the legacy default stream) while one is set, else the context's
  // own stream (the synchronous host API).
  void set_stream(cudaStream_t s) { user_stream_ = s; has_user_stream_ = true; }
  void clear_stream() { user_stream_ = nullptr; has_user_stream_ = false; }
  cudaStream_t exec_stream() const { return has_user_stream_ ? user_stream_ : stream_; }
  cudaStream_t own_stream() const { return stream_; }
  bool has_user_stream() const { return has_user_stream_; }

  Status plan(const Dims& work, const PlanEntry** out);
  Status workspace(const PlanEntry& pe, const Dims& img, const Dims& ker,
                   Workspace** out);
  // Workspace of batch slot `slot` (one per volume of a batched call).
  Status workspace_slot(int slot, const PlanEntry& pe, const Dims& img, const Dims& ker,
                        Workspace** out);
  // Stream i of the batch stream pool (created on first use).
  Status batch_stream(int i, cudaStream_t* out);
  // Instantiated CUDA graph of a batched call, looked up by the call's
  // pointers and sizes (nullptr when absent); add_graph takes ownership.
  cudaGraphExec_t find_graph(const std::vector<unsigned long long>& key) const;
  void add_graph(std::vector<unsigned long long> key, cudaGraphExec_t g);
  // With autotuning on, the first plan of a work box times the planner's
  // candidate tilings on the device and keeps the fastest.
  void set_autotune(bool on) { autotune_ = on; }
  bool autotune() const { return autotune_; }
  void release_workspaces();
  // One growable device block for auxiliary scratch (the learned-start
  // network's weights and activations); freed by release_workspaces.
  Status aux_scratch(size_t bytes, void** out);
  // Queue and tables of the persistent batched launch.  Captured graphs use
  // it, so growing it first drops every cached graph.
  Status batch_scratch(size_t bytes, void** out);
  // Reads and clears the error word (no synchronisation: it reports what
  // kernels that have finished recorded).
  Status check_device_errors();

  std::mutex mu;  // serialises API calls on this context

 private:
  int device_;
  cudaStream_t stream_ = nullptr;
  int* err_host_ = nullptr;  // mapped pinned host memory
  int* err_dev_ = nullptr;
  void* aux_ = nullptr;
  size_t aux_cap_ = 0;
  void* bq_ = nullptr;
  size_t bq_cap_ = 0;
  cudaStream_t user_stream_ = nullptr;
  bool has_user_stream_ = false;
  Status build_entry(const VolPlan& P, std::unique_ptr<PlanEntry>* out);
  Status tune(const Dims& wd, std::unique_ptr<PlanEntry>* out);
  // keyed by the work box and whether the autotuner chose the plan
  std::map<std::tuple<int, int, int, int>, std::unique_ptr<PlanEntry>> plans_;
  Workspace ws_;
  std::vector<std::unique_ptr<Workspace>> slots_;
  std::vector<cudaStream_t> bstreams_;
  struct GraphEntry {
    std::vector<unsigned long long> key;
    cudaGraphExec_t exec;
  };
  std::vector<GraphEntry> graphs_;
  bool autotune_ = false;
};

// ----------------------------------------------------------- algorithms
// All take unpadded device volumes and write the clipped result to a device
// buffer of imageDim voxels.  They enqueue on ctx.exec_stream() only.
Status run_convolve(Context& ctx, const float* img, Dims id, const float* ker,
                    Dims kd, float* out);
Status run_wiener(Context& ctx, const float* img, Dims id, const float* ker,
                  Dims kd, float* out, float eps);
// Circular correlation with the kernel (the conjugated OTF in the z pass).
Status run_correlate(Context& ctx, const float* img, Dims id, const float* ker, Dims kd,
                     float* out);
// Richardson-Lucy whose second convolution per iteration is a correlation
// with the kernel (conjugated OTF).
Status run_rl_correlate(Context& ctx, const float* img, Dims id, const float* ker, Dims kd,
                        float* out, int iters);
Status run_rl(Context& ctx, const float* img, Dims id, const float* ker,
              Dims kd, float* out, int iters);
// Richardson-Lucy from a given first estimate (image-sized, nullptr: the
// image) with an optional I-divergence trace idiv[0..iters) (device doubles:
// the image against h * the estimate at the start of each iteration).
Status run_rl_ex(Context& ctx, const float* img, Dims id, const float* ker, Dims kd,
                 const float* start, float* out, int iters, double* idiv);
// Accelerated Richardson-Lucy (Biggs-Andrews vector extrapolation) from
// `start` (image-sized; nullptr: the image), optional I-divergence trace as
// run_rl_ex (entries k < iters at the extrapolated points).
Status run_rl_accel(Context& ctx, const float* img, Dims id, const float* ker, Dims kd,
                    const float* start, float* out, int iters, double* idiv);
// I-divergence restoration after Markham and Conchello (conjugate gradients
// on s = a^2 with an exact quadratic line model); alpha weights sum s^2.
Status run_idiv_cg(Context& ctx, const float* img, Dims id, const float* ker, Dims kd,
                   float* out, int iters, float alpha);
// Blind ML with the PSF update (alternating object and PSF steps; psf_out
// optional, on the kernel's grid).
Status run_blind_psf(Context& ctx, const float* img, Dims id, const float* ker, Dims kd,
                     float* out, float* psf_out, int iters, int psf_subiters);
// uint16 <-> float casts of the raw-image path (x86 conversion semantics out).
Status cast_u16_to_f32(Context& ctx, const uint16_t* a, float* b, long long n);
Status cast_f32_to_u16(Context& ctx, const float* a, uint16_t* b, long long n);
// Richardson-Lucy on n independent volumes of any sizes (device pointers):
// each volume has its own plan and workspace, volumes run concurrently on the
// batch stream pool, and with use_graph the whole batch is captured into one
// CUDA graph (replayed when the same batch is run again).
// persistent: the iterations of all volumes run in one persistent launch
// (kern_batch.cu) instead of per-volume launches on a pool of streams.
Status run_rl_batch(Context& ctx, int n, const float* const* imgs, const Dims* ids,
                    const float* const* kers, const Dims* kds, float* const* outs, int iters,
                    bool use_graph, bool persistent = false);
// The persistent launch (kern_batch.cu): scratch holds batch_queue_bytes(n,
// iters) bytes; the volumes' set-up (OTF, energy, first forward transform)
// is already enqueued on st.
size_t batch_queue_bytes(int n, int iters);
Status launch_rl_batch(Context& ctx, int n, const PlanEntry* const* pes, Workspace* const* wss,
                       const float* const* imgs, const Dims* ids, const Dims* wds, int iters,
                       void* scratch, cudaStream_t st);
Status run_blind(Context& ctx, const float* img, Dims id, const float* ker,
                 Dims kd, float* out, int iters);
Status run_jvc(Context& ctx, const float* img, Dims id, const float* ker,
               Dims kd, float* out, int iters, float image_max,
               const float* smooth_sigma, int smooth_interval);
// Learned start (nn.cu): RL `pre` iterations, the 3-D U-Net's prediction from
// that iterate (FP32 parameter vector `params` of nn_param_count() floats, on
// the device), RL resumed from the prediction for `post` iterations; idiv as
// run_rl_ex for the resumed part.  Image dimensions must be multiples of 8.
long long nn_param_count();
Status run_ml_learned(Context& ctx, const float* img, Dims id, const float* ker, Dims kd,
                      const float* params, int pre, float* out, int post, double* idiv);
// The network's prediction alone: out = max(0, m ((x/m + 0.01) e^r - 0.01)),
// r = U-Net(log(x/m + 0.01)), m = mean(x); x and out are D x H x W volumes.
Status nn_predict(Context& ctx, const float* params, const float* x, int D, int H, int W,
                  float* out);
// Failure-detection self test: enqueues a one-thread kernel whose bounded
// mbarrier wait runs out (no copy is issued) and records a timeout in the
// context's error word, as a fused pass would.
Status inject_wait_timeout(Context& ctx);
// FP64 I-divergence of g against ghat (both unpadded device volumes).
Status run_idivergence(Context& ctx, const float* g, const float* ghat,
                       long long n, double* result);

Context* global_context();  // nullptr when not registered
void set_last_error(const char* msg);

// ------------------------------------------------ launch accounting
// Counts every kernel launch of the library (for benchmarks) and, when
// timing is enabled, records a CUDA event pair around each fused-pass launch
// on the launching stream.
void note_launch_begin(int kind, cudaStream_t st);
void note_launch_end(int kind, cudaStream_t st);
void set_capturing(bool on);
bool pdl_enabled();
// cudaFuncSetAttribute(MaxDynamicSharedMemorySize) for kernels above 48 KB,
// issued once per kernel, device and size (the attribute call is not free, and
// a solve launches each kernel hundreds of times).
cudaError_t smem_opt_in(const void* kernel, int smem);
long long launch_count();
// Counts one kernel launch that note_launch_begin/end do not bracket.
void count_launch();
int static_family_mask();
// DFT precision mode of the specialised z pass (0 FP32 register passes, 1
// split hi+lo FP16 tensor-core first z stage, 2 the same in BF16); applies
// to shapes with a 16 x 16 z axis (the 1024 x 1024 x 256 box).
void set_dft_precision(int mode);
int dft_precision();
void timing_enable(bool on);
// Synchronises the recorded events and returns per-kind totals (ms) and
// counts; clears the record.
void timing_collect(double* ms, long long* counts);

}  // namespace clarity
