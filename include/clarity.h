/*
 * clarity.h -- public C ABI of the B200-native Clarity deconvolution library.
 *
 * This header declares the same entry points, argument order, types and
 * result-code values as the reference library's public header
 * (Clarity.h.in), so that an existing caller can relink against
 * libclarity.so without source changes.  Every pointer argument is HOST
 * memory owned by the caller; every call is synchronous (the result is in
 * the caller's buffer when the call returns).  Work runs on CUDA device 0
 * (or the device set with clarityx_set_device) on hand-written sm_100a
 * kernels; there is no CPU fallback.
 *
 * Reference interface each declaration replaces is cited as
 * Clarity.h.in:<line> (declaration) and src/<file>:<line> (definition).
 */
#ifndef CLARITY_B200_CLARITY_H_
#define CLARITY_B200_CLARITY_H_

#ifdef __cplusplus
#define CLARITY_API extern "C" __attribute__((visibility("default")))
#else
#define CLARITY_API __attribute__((visibility("default")))
#endif

/* Library version 1.1.0 flattened, as the reference's CLARITY_VERSION
 * (Clarity.h.in:41, CMakeLists.txt:27-31). */
#define CLARITY_VERSION 110

/* Result codes.  The numeric values are part of the ABI and follow the
 * reference enum order exactly (Clarity.h.in:90-101): success is 5. */
typedef enum {
  CLARITY_FFT_FAILED = 0,           /* an FFT stage could not run          */
  CLARITY_OUT_OF_MEMORY = 1,        /* host allocation failed              */
  CLARITY_DEVICE_OUT_OF_MEMORY = 2, /* device allocation failed            */
  CLARITY_INVALID_OPERATION = 3,    /* no usable device, or a device failure */
  CLARITY_INVALID_ARGUMENT = 4,     /* NULL pointer or dimension <= 0      */
  CLARITY_SUCCESS = 5
} ClarityResult_t;

/* Volume dimensions, x fastest in memory: index = (z*y_dim + y)*x_dim + x
 * (Clarity.h.in:110-114; layout from src/ImageClip.cxx:41-42). */
typedef struct _Clarity_Dim3_t {
  int x;
  int y;
  int z;
} Clarity_Dim3;

/* Clarity.h.in:123-125; src/Clarity.cxx:106-113. */
CLARITY_API Clarity_Dim3 Clarity_Dim3FromArray(int dimArray[3]);

/* Reference-counted initialisation (Clarity.h.in:137-139;
 * src/Clarity.cxx:46-79).  The first call selects the CUDA device and
 * creates the library context; later calls only bump the count.  Returns
 * CLARITY_INVALID_OPERATION when no usable sm_100 device is present.
 * As with the reference, calling it is optional: a call made without a
 * registration creates the context itself (the reference's own raw-image
 * app never registers), and a later Clarity_Register adopts that context. */
CLARITY_API ClarityResult_t Clarity_Register(void);

/* Clarity.h.in:147-149; src/Clarity.cxx:82-91.  The last call releases
 * every device buffer, plan and stream the library holds. */
CLARITY_API ClarityResult_t Clarity_UnRegister(void);

/* Clarity.h.in:160-162; src/Clarity.cxx:93-103.  Sets the host thread count
 * used by the host-side pad/clip helpers; device work is unaffected. */
CLARITY_API ClarityResult_t Clarity_SetNumberOfThreads(unsigned n);

/* Cyclic shift of src into a dst box filled with fillValue
 * (Clarity.h.in:181-185; src/ImagePadSpatialShift.cxx:32-69).  Host
 * buffers; runs on the host like the reference. */
CLARITY_API ClarityResult_t Clarity_ImagePadSpatialShift(
    float *dst, Clarity_Dim3 dstDim, float *src, Clarity_Dim3 srcDim,
    int shift[3], float fillValue);

/* Crop from the origin (Clarity.h.in:200-202; src/ImageClip.cxx:30-50). */
CLARITY_API ClarityResult_t Clarity_ImageClip(
    float *dst, Clarity_Dim3 dstDim, float *src, Clarity_Dim3 srcDim);

/* Clarity.h.in:210-212; src/Clarity.cxx:116-150.  Returns a static string. */
CLARITY_API char *Clarity_ResultString(ClarityResult_t result);

/* Wiener filter U = conj(H) G / (|H|^2 + epsilon) / N on the padded work box
 * (Clarity.h.in:236-240; src/WienerDeconvolve.cxx:211-290,48-66). */
CLARITY_API ClarityResult_t Clarity_WienerDeconvolve(
    float *inImage, Clarity_Dim3 imageDim, float *kernelImage,
    Clarity_Dim3 kernelDim, float *outImage, float epsilon);

/* Jansen-van Cittert (Clarity.h.in:257-261;
 * src/JansenVanCittertDeconvolve.cxx:311-389).  iterations <= 1 performs
 * exactly one update, as the reference does (:167-173). */
CLARITY_API ClarityResult_t Clarity_JansenVanCittertDeconvolve(
    float *inImage, Clarity_Dim3 imageDim, float *kernelImage,
    Clarity_Dim3 kernelDim, float *outImage, int iterations);

/* Jansen-van Cittert with a Gaussian smoothing of the estimate every
 * smoothInterval iterations (Clarity.h.in:285-291).  The reference body is
 * a stub that writes zeros (src/SmoothedJansenVanCittertDeconvolve.cxx:27-40);
 * this library implements the documented intent: smoothSigma[d] points to
 * the Gaussian sigma (voxels) along axis d (x, y, z); a NULL smoothSigma or
 * smoothInterval == 0 disables smoothing (plain JVC). */
CLARITY_API ClarityResult_t Clarity_SmoothedJansenVanCittertDeconvolve(
    float *inImage, Clarity_Dim3 imageDim, float *kernelImage,
    Clarity_Dim3 kernelDim, float *outImage, unsigned iterations,
    unsigned smoothInterval, float *smoothSigma[3]);

/* Clarity.h.in:314-319.  The reference body writes zeros
 * (src/IDivergenceDeconvolve.cxx:59-72); this library does the same, so the
 * ABI is complete.  The I-divergence functional itself is available as
 * clarityx_idivergence (clarity_ext.h). */
CLARITY_API ClarityResult_t Clarity_IDivergenceDeconvolve(
    float *inImage, Clarity_Dim3 imageDim, float *kernelImage,
    Clarity_Dim3 kernelDim, float *outImage);

/* Richardson-Lucy / maximum likelihood with per-iteration flux rescaling
 * (Clarity.h.in:337-341; src/MaximumLikelihoodDeconvolve.cxx:255-332,48-81).
 * iterations <= 0 returns the input image unchanged (the reference leaves
 * the output unwritten in that case). */
CLARITY_API ClarityResult_t Clarity_MaximumLikelihoodDeconvolve(
    float *inImage, Clarity_Dim3 imageDim, float *kernelImage,
    Clarity_Dim3 kernelDim, float *outImage, int iterations);

/* Blind maximum likelihood with the reference's CPU semantics
 * (Clarity.h.in:358-363; src/BlindMaximumLikelihoodDeconvolve.cxx:249-317,
 * 50-148): the kernel guess is normalised to unit sum and the image is
 * updated by u' = u (h * (g / (h * u))) with no flux rescale; the kernel
 * itself is not updated (the reference's update line :96 is disabled). */
CLARITY_API ClarityResult_t Clarity_BlindMaximumLikelihoodDeconvolve(
    float *inImage, Clarity_Dim3 imageDim, float *kernelImage,
    Clarity_Dim3 kernelDim, float *outImage, int iterations);

/* Circular convolution on the padded work box, clipped back to imageDim
 * (Clarity.h.in:379-383; src/Convolve.cxx:41-115,146-184). */
CLARITY_API ClarityResult_t Clarity_Convolve(
    float *inImage, Clarity_Dim3 imageDim, float *kernel,
    Clarity_Dim3 kernelDim, float *outImage);

#endif /* CLARITY_B200_CLARITY_H_ */
