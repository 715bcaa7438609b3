/* fftw3.h -- TEST INFRASTRUCTURE ONLY (oracle).
 *
 * Declares the nine FFTW 3 single-precision entry points the reference calls
 * (src/FFT.cxx:80-86,131-137; src/Clarity.cxx:49,86,100;
 * src/Memory.cxx:59,85,204) so the reference sources compile unchanged
 * against this project's own CPU FFT (fftw_shim.cpp).  FFTW itself is not
 * installed here; the names, argument order and the FFTW_ESTIMATE flag value
 * must match FFTW's public API because the reference calls them by name. */
#ifndef CLARITY_ORACLE_FFTW3_SHIM_H_
#define CLARITY_ORACLE_FFTW3_SHIM_H_
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef float fftwf_complex[2];
typedef struct fftwf_plan_s *fftwf_plan;

#define FFTW_ESTIMATE (1U << 6)

fftwf_plan fftwf_plan_dft_r2c_3d(int n0, int n1, int n2, float *in,
                                 fftwf_complex *out, unsigned flags);
fftwf_plan fftwf_plan_dft_c2r_3d(int n0, int n1, int n2, fftwf_complex *in,
                                 float *out, unsigned flags);
void fftwf_execute(const fftwf_plan plan);
void fftwf_destroy_plan(fftwf_plan plan);
void *fftwf_malloc(size_t n);
void fftwf_free(void *p);
int fftwf_init_threads(void);
void fftwf_cleanup_threads(void);
void fftwf_plan_with_nthreads(int nthreads);

#ifdef __cplusplus
}
#endif
#endif
