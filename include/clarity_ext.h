/*
 * clarity_ext.h -- extensions of the Clarity C ABI (no counterpart in the
 * reference's public header).  Device-pointer entry points let a caller keep
 * volumes resident in HBM across calls (the public Clarity_* functions take
 * host buffers and copy in and out on every call); the rest are diagnostics
 * and host-side fault injection for tests.
 *
 * Device-pointer functions: every pointer is a CUDA device pointer on the
 * library's device; `stream` is a cudaStream_t and work is enqueued on it
 * (NULL is the legacy default stream, so the work is ordered with the
 * caller's other default-stream work).  They are asynchronous with respect to
 * the host unless stated.
 *
 * Failure detection: the fused passes wait for their tile copies with
 * bounded waits.  A wait that gives up records the failure in the library's
 * error word (mapped host memory, readable without synchronising) and the
 * kernel returns.  clarityx_synchronize reports it; so does the next call
 * into the library, which then returns CLARITY_INVALID_OPERATION without
 * enqueuing anything (the failed call's result is not valid).  The word is
 * cleared once reported.
 */
#ifndef CLARITY_B200_CLARITY_EXT_H_
#define CLARITY_B200_CLARITY_EXT_H_

#include <stdint.h>

#include "clarity.h"

/* Message of the last failing call on this thread's library state, or "". */
CLARITY_API const char *clarityx_last_error(void);

/* CUDA device used by the next Clarity_Register that creates the context
 * (default 0).  Returns CLARITY_INVALID_OPERATION once registered. */
CLARITY_API ClarityResult_t clarityx_set_device(int device);

/* Host-side fault injection for tests: the countdown-th device allocation
 * from now fails as if cudaMalloc had run out of memory (0 disables). */
CLARITY_API void clarityx_inject_device_alloc_failure(int countdown);

/* Releases cached work buffers (plans stay cached). */
CLARITY_API ClarityResult_t clarityx_trim(void);

/* Blocks until `stream` has finished (NULL: every stream of the library's
 * device, the library's own included), then returns the first asynchronous
 * error as a result code: a CUDA error, or CLARITY_INVALID_OPERATION when a
 * device-side bounded wait gave up (see above). */
CLARITY_API ClarityResult_t clarityx_synchronize(void *stream);

/* Failure-detection self test: enqueues on `stream` a one-thread kernel that
 * arms an mbarrier for bytes no copy will deliver and waits on it with a
 * short bound (about a millisecond).  The wait gives up and records a
 * timeout exactly as a fused pass's would, so the next clarityx_synchronize
 * or library call reports CLARITY_INVALID_OPERATION.  No copy is issued and
 * the GPU stays usable.  For tests of callers' error handling. */
CLARITY_API ClarityResult_t clarityx_inject_wait_timeout(void *stream);

/* Device-resident versions of the public algorithms.  image/kernel/out are
 * unpadded device volumes of imageDim / kernelDim / imageDim voxels. */
CLARITY_API ClarityResult_t clarityx_convolve_device(
    const float *image, Clarity_Dim3 imageDim, const float *kernel,
    Clarity_Dim3 kernelDim, float *out, void *stream);
CLARITY_API ClarityResult_t clarityx_wiener_device(
    const float *image, Clarity_Dim3 imageDim, const float *kernel,
    Clarity_Dim3 kernelDim, float *out, float epsilon, void *stream);
CLARITY_API ClarityResult_t clarityx_ml_device(
    const float *image, Clarity_Dim3 imageDim, const float *kernel,
    Clarity_Dim3 kernelDim, float *out, int iterations, void *stream);
/* Conjugate-for-correlation opt-ins (no reference counterpart; the
 * reference never conjugates the OTF, src/MaximumLikelihoodDeconvolve.cxx
 * :57,65 and src/ModulateGPU.cu:63-72).  clarityx_correlate_device is
 * clarityx_convolve_device with the kernel's spectrum conjugated in the z
 * pass: the circular correlation with the kernel.
 * clarityx_ml_correlate_device is clarityx_ml_device whose second
 * convolution per iteration (the reference's h * (g / (h * u))) is that
 * correlation -- the h^T of the textbook Richardson-Lucy update.  The two
 * forms agree for a kernel symmetric about its centre; for the 256x256x64
 * halo PSF (|Im H| / |H| ~ 1e-4) they differ by more than the reference
 * parity tolerance, so the reference form stays the default. */
CLARITY_API ClarityResult_t clarityx_correlate_device(
    const float *image, Clarity_Dim3 imageDim, const float *kernel,
    Clarity_Dim3 kernelDim, float *out, void *stream);
CLARITY_API ClarityResult_t clarityx_ml_correlate_device(
    const float *image, Clarity_Dim3 imageDim, const float *kernel,
    Clarity_Dim3 kernelDim, float *out, int iterations, void *stream);

/* Blind ML with the PSF update that Clarity_BlindMaximumLikelihoodDeconvolve
 * leaves disabled (src/BlindMaximumLikelihoodDeconvolve.cxx:96): per outer
 * iteration one object step o <- o (h * (g / (h * o))), then
 * psf_subiterations PSF steps h <- h (o * (g / (h * o))) renormalised to unit
 * sum.  psf_out (optional, kernelDim voxels) receives the PSF estimate on the
 * kernel's grid.  No reference counterpart; device pointers, asynchronous. */
CLARITY_API ClarityResult_t clarityx_blind_ml_psf_device(
    const float *image, Clarity_Dim3 imageDim, const float *kernel,
    Clarity_Dim3 kernelDim, float *out, float *psf_out, int iterations,
    int psf_subiterations, void *stream);

/* I-divergence restoration after J. Markham and J.A. Conchello, J. Opt. Soc.
 * Am. A 18(5), 2001: the method Clarity_IDivergenceDeconvolve declares
 * (Clarity.h.in:294-319), whose reference body is a stub that writes zeros
 * (src/IDivergenceDeconvolve.cxx).  Minimises sum g ln(g/gh) + gh - g +
 * alpha sum s^2 with gh = kernel * s over the padded work box, s = a^2 >= 0,
 * by `iterations` Polak-Ribiere conjugate-gradient steps on a from
 * a = sqrt(image), each with an exact quadratic line model and four Newton
 * steps.  alpha >= 0.  Device pointers, asynchronous on `stream`. */
CLARITY_API ClarityResult_t clarityx_idiv_deconvolve_device(
    const float *image, Clarity_Dim3 imageDim, const float *kernel,
    Clarity_Dim3 kernelDim, float *out, int iterations, float alpha, void *stream);

/* Clarity_MaximumLikelihoodDeconvolve on uint16 host volumes, as the
 * reference's DeconvolveRawImages app does around it
 * (apps/DeconvolveRawImages/DeconvolveRawImages.cxx:91-116), with the casts on
 * the device: only uint16 data crosses the bus.  The result is converted as
 * static_cast<unsigned short>(float) behaves on x86 (truncation to a 32-bit
 * integer, low 16 bits), so the output is bit-identical to casting this
 * library's float result on the host.  Synchronous. */
CLARITY_API ClarityResult_t clarityx_ml_u16(const uint16_t *image, Clarity_Dim3 imageDim,
                                            const uint16_t *kernel, Clarity_Dim3 kernelDim,
                                            uint16_t *out, int iterations);

/* Richardson-Lucy (Clarity.h.in:337-341) resumed from `start`, an estimate of
 * imageDim voxels on the device (NULL: the image, as the reference), with an
 * optional I-divergence trace: when idiv is not NULL, idiv[k] (device doubles,
 * `iterations` + 1 of them) receives sum g ln(g/b) + b - g over the image, b =
 * kernel * (the estimate at the start of iteration k), accumulated in FP64 by
 * the ratio pass at no extra pass over memory; idiv[iterations] is the
 * result's own (one more convolution). */
CLARITY_API ClarityResult_t clarityx_ml_ex_device(
    const float *image, Clarity_Dim3 imageDim, const float *kernel,
    Clarity_Dim3 kernelDim, const float *start, float *out, int iterations,
    double *idiv, void *stream);

/* Accelerated Richardson-Lucy: the update and flux rescale of
 * Clarity_MaximumLikelihoodDeconvolve applied at extrapolated points
 * y = max(0, x + alpha (x - x_prev)), alpha from the last two steps (vector
 * extrapolation of Biggs and Andrews, Applied Optics 36(8):1766-1775, 1997).
 * No reference counterpart.  start and idiv as clarityx_ml_ex_device (trace
 * entries before the last taken at the extrapolated points). */
CLARITY_API ClarityResult_t clarityx_ml_accel_device(
    const float *image, Clarity_Dim3 imageDim, const float *kernel,
    Clarity_Dim3 kernelDim, const float *start, float *out, int iterations,
    double *idiv, void *stream);

/* Richardson-Lucy on `count` independent volumes of any sizes (device
 * pointers, one kernel per volume): each volume has its own plan and
 * workspace and the volumes run concurrently on a pool of streams, forked
 * from and joined back to `stream`.  flags & CLARITYX_BATCH_GRAPH captures the
 * whole batch into one CUDA graph, kept and replayed when the same batch
 * (same pointers, sizes and iterations) is run again.
 * flags & CLARITYX_BATCH_PERSISTENT runs the iterations of all volumes in one
 * persistent launch: a fixed grid of blocks takes tiles of every volume's
 * passes from one work queue (each volume's set-up and its clipped result
 * are ordinary launches around it).  The iterations then use the
 * runtime-planned pass kernels for every work box, so a box that has
 * specialised kernels can differ from its single-volume solve in the last
 * bits.  Asynchronous like the other _device calls.  Extension of
 * Clarity_MaximumLikelihoodDeconvolve (Clarity.h.in:337-341), which takes
 * one volume. */
#define CLARITYX_BATCH_GRAPH 1
#define CLARITYX_BATCH_PERSISTENT 2
CLARITY_API ClarityResult_t clarityx_ml_batch_device(
    int count, const float *const *images, const Clarity_Dim3 *imageDims,
    const float *const *kernels, const Clarity_Dim3 *kernelDims,
    float *const *outs, int iterations, int flags, void *stream);

/* Autotuning of work-box plans (off by default): with it on, the first use of
 * a work box times the planner's best candidate tilings (one RL iteration's
 * passes each) and keeps the fastest. */
CLARITY_API void clarityx_autotune(int on);

/* Precision form of the 3-D FFT (no reference counterpart; the reference
 * calls FFTW/cuFFT in FP32).  0 (default): every DFT stage in FP32 register
 * passes.  1: the first radix-16 stage of the z axis (forward and inverse)
 * as tensor-core GEMMs on split hi+lo FP16 operands with FP32 accumulation,
 * each 8-line tile scaled by a power of two into FP16's range -- FP32-class
 * accuracy.  2: the same on split hi+lo BF16 operands (no scaling, about
 * 2^-16 relative per stage).  It applies to work boxes whose specialised z
 * pass has a 16 x 16 z axis (the 1024 x 1024 x 256 box of a 512 x 512 x 128
 * image with a same-size kernel); other boxes, and every OTF, stay FP32.
 * Process-wide; returns CLARITY_INVALID_ARGUMENT for other modes. */
CLARITY_API ClarityResult_t clarityx_set_dft_precision(int mode);
CLARITY_API int clarityx_dft_precision(void);

CLARITY_API ClarityResult_t clarityx_blind_ml_device(
    const float *image, Clarity_Dim3 imageDim, const float *kernel,
    Clarity_Dim3 kernelDim, float *out, int iterations, void *stream);
CLARITY_API ClarityResult_t clarityx_jvc_device(
    const float *image, Clarity_Dim3 imageDim, const float *kernel,
    Clarity_Dim3 kernelDim, float *out, int iterations, void *stream);

/* I-divergence sum_i g ln(g/ghat) + ghat - g (alpha = 0 form of
 * src/IDivergenceDeconvolve.cxx:33-47), accumulated in FP64; 0 ln 0 = 0 and
 * voxels with g > 0 and ghat <= 0 are skipped.  Host buffers; synchronous. */
CLARITY_API ClarityResult_t clarityx_idivergence(const float *g,
                                                 const float *ghat,
                                                 long long n, double *result);

/* Plan chosen for a padded work box: fills up to 16 ints
 * {M, XS, Ay, By, G, W, KG, xy_blocks, z_blocks, xy_smem, z_smem,
 *  x passes, y0 passes, z passes, xmode, spec_elems / 1024}.
 * Returns CLARITY_INVALID_ARGUMENT for shapes the planner rejects.  Needs
 * no device. */
CLARITY_API ClarityResult_t clarityx_plan_info(Clarity_Dim3 workDim,
                                               int *fields, int nfields);

/* Circular convolution of device buffers that allocates nothing (no
 * cudaMalloc, cudaFree or allocating library call; no Clarity_Register
 * needed).  It has no counterpart in the reference.  It is for callers that
 * cannot allocate device memory once running: code that runs under a memory
 * pool it manages itself (an allocation behind the pool's back breaks its
 * accounting), real-time loops whose footprint must be fixed up front (an
 * allocation can stall or fail mid-run), and plugins hosted in a context
 * that forbids cudaMalloc.
 * image/kernel/out are device buffers on the current device, as in
 * clarityx_convolve_device, and the result is the same.  Work is enqueued
 * on `stream` (NULL: the legacy default stream, as for every _device call);
 * no library stream or registration is involved.
 * Scratch: one 32 MiB array in the library's device memory (held by every
 * GPU that loads the library until exit).  The limit is in bytes: the work
 * box (image + kernel per axis) fits when its OTF and work spectrum
 * (2 x spec_elems x 8 bytes; spec_elems is field 15 of clarityx_plan_info,
 * in units of 1024) plus the plan tables fit in 32 MiB -- a 64^3 image with a
 * 64^3 kernel (work box 128^3, 16.5 MiB) fits, 128 x 128 x 192 (24.4 MiB)
 * fits, 256 x 256 x 256 does not.  A box that does not fit returns
 * CLARITY_INVALID_ARGUMENT with the size needed in clarityx_last_error().
 * The first call on each device looks up the array's device address
 * (cudaGetSymbolAddress, with that device current) and keeps it for the
 * life of the process: make that first call before any stream capture, and
 * do not use this entry point after cudaDeviceReset.  Every call shares the
 * one array: calls that overlap on the GPU (two streams, two host threads)
 * race and corrupt each other's results, so serialise them.  Nothing in the
 * array needs to start at zero; each call rewrites what it reads. */
CLARITY_API ClarityResult_t clarityx_convolve_noalloc(
    const float *image, Clarity_Dim3 imageDim, const float *kernel,
    Clarity_Dim3 kernelDim, float *out, void *stream);

/* Learned-start network kernels (clarity_b200/unet.py builds the network on
 * them).  Device pointers; activations are BF16 [v][c] with v = (z*H + y)*W +
 * x, weights BF16 [cout][27][cin] with tap = (dz+1)*9 + (dy+1)*3 + (dx+1),
 * accumulation FP32.  Channel counts of conv3/conv3_wgrad are multiples of 16;
 * buffers 16-byte aligned.  No reference counterpart.
 *
 * conv3: y = act(bias + 3x3x3 convolution, zero padding) of x1 [D,H,W,c1]
 *   concatenated with x2 [D/2,H/2,W/2,c2] read through nearest upsampling (x2
 *   may be NULL, c2 = 0); act = ReLU when relu, then y *= (mask > 0) when mask
 *   is given.  Tensor cores, BF16 operands, FP32 accumulation: tcgen05 with
 *   tensor-memory accumulators when W is a multiple of 32 (unless the
 *   environment sets CLARITY_NN_TCGEN05=0), else mma.sync.
 * conv3_wgrad: dw[cout][27][cin] += sum_v dy[v][co] in(v + tap)[ci], dbias[co]
 *   += sum_v dy[v][co] (FP32, accumulated: zero them first).
 * conv_in / conv_in_wgrad: the 1 -> 16 first layer (float input, FP32
 *   weights [16][27]), ReLU output.
 * head / head_loss_grad: r = b + sum_c w[c] y[v][c] over 16 channels; the loss
 *   mean (r - t)^2 added to *loss, its gradient dy (masked by y > 0), dw, db.
 * pool2: 2x2x2 average pool.  merge_skip_grad: (dxcat[.., 0:c] + dp/8
 *   upsampled) * (s > 0).  up_grad: 2x2x2 sums of dxcat[.., c1:c1+c2] masked by
 *   coarse > 0.  adam: one bias-corrected Adam step.  pack_weights: BF16
 *   forward weights and the mirrored, transposed backward-data weights from the
 *   FP32 master copy. */
CLARITY_API ClarityResult_t clarityx_nn_conv3(const void *x1, int c1, const void *x2, int c2,
                                              int D, int H, int W, const void *w,
                                              const float *bias, int cout, int relu,
                                              const void *mask, void *y, void *stream);
CLARITY_API ClarityResult_t clarityx_nn_conv3_wgrad(const void *x1, int c1, const void *x2,
                                                    int c2, int D, int H, int W, const void *dy,
                                                    int cout, float *dw, float *dbias,
                                                    void *stream);
CLARITY_API ClarityResult_t clarityx_nn_conv_in(const float *x, int D, int H, int W,
                                                const float *w, const float *b, void *y,
                                                void *stream);
CLARITY_API ClarityResult_t clarityx_nn_conv_in_wgrad(const float *x, int D, int H, int W,
                                                      const void *dy, float *dw, float *db,
                                                      void *stream);
CLARITY_API ClarityResult_t clarityx_nn_head(const void *y, long long V, const float *w,
                                             const float *b, float *r, void *stream);
CLARITY_API ClarityResult_t clarityx_nn_head_loss_grad(const void *y, long long V,
                                                       const float *w, const float *r,
                                                       const float *t, void *dy, float *dw,
                                                       float *db, double *loss, void *stream);
CLARITY_API ClarityResult_t clarityx_nn_pool2(const void *x, int C, int D, int H, int W,
                                              void *y, void *stream);
CLARITY_API ClarityResult_t clarityx_nn_merge_skip_grad(const void *dxcat, int ccat,
                                                        const void *dp, const void *s, int c,
                                                        int D, int H, int W, void *out,
                                                        void *stream);
CLARITY_API ClarityResult_t clarityx_nn_up_grad(const void *dxcat, int ccat, int c1, int c2,
                                                const void *coarse, int D, int H, int W,
                                                void *out, void *stream);
CLARITY_API ClarityResult_t clarityx_nn_adam(float *p, const float *g, float *m, float *v,
                                             long long n, float lr, float b1, float b2,
                                             float eps, int step, void *stream);
CLARITY_API ClarityResult_t clarityx_nn_pack_weights(const float *w, int cout, int cin,
                                                     void *wf, void *wb, void *stream);

/* Learned start as one call (no reference counterpart): RL `pre` iterations
 * (clarityx_ml_device), the learned-start network's prediction of an advanced
 * estimate from that iterate, then RL resumed from the prediction for `post`
 * iterations (clarityx_ml_ex_device with a start; idiv as there, post + 1
 * entries).  The network is the 3-D U-Net the kernels below implement (4
 * levels, widths 16-32-64-128, BF16 tensor-core convolutions, FP32
 * accumulation); `params` is its FP32 parameter vector on the device,
 * nparams = clarityx_nn_param_count() floats in the order of
 * clarity_b200/unet.py (clarity_b200/learned_start_weights.npy holds trained
 * ones).  Around the network the estimate is taken to the log domain and
 * back inside its first and last kernels: input log(x/m + 0.01), prediction
 * max(0, m ((x/m + 0.01) e^r - 0.01)) with m = mean(x).  Image dimensions
 * must be multiples of 8.  Device pointers, asynchronous on `stream`. */
CLARITY_API ClarityResult_t clarityx_ml_learned_device(
    const float *image, Clarity_Dim3 imageDim, const float *kernel,
    Clarity_Dim3 kernelDim, const float *params, long long nparams, int pre,
    float *out, int post, double *idiv, void *stream);
/* The network's prediction alone: out = max(0, m ((x/m + 0.01) e^r - 0.01)),
 * r = U-Net(log(x/m + 0.01)), for a volume x of `dim` voxels (multiples of
 * 8).  Needs Clarity_Register (its activations live in the library's
 * cached scratch). */
CLARITY_API ClarityResult_t clarityx_nn_predict(const float *params, long long nparams,
                                                const float *x, Clarity_Dim3 dim, float *out,
                                                void *stream);
/* Length of the network's FP32 parameter vector. */
CLARITY_API long long clarityx_nn_param_count(void);

/* Benchmark probes.  clarityx_launch_count: kernels the library has
 * launched so far.  clarityx_timing_enable(1) makes every fused-pass launch
 * record a CUDA event pair on its stream; clarityx_timing_collect waits for
 * them and returns, per kernel family (0 xy-forward, 1 z, 2 xy-inverse+forward,
 * 3 xy-inverse, 4 other, 5 xy-inverse+forward of the RL product step), the
 * summed milliseconds and launch counts, then clears the record. */
CLARITY_API long long clarityx_launch_count(void);
CLARITY_API void clarityx_timing_enable(int on);
CLARITY_API void clarityx_timing_collect(double *ms, long long *counts, int n);

#endif /* CLARITY_B200_CLARITY_EXT_H_ */
