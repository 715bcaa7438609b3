// fftw_shim.cpp -- TEST INFRASTRUCTURE ONLY (oracle).
//
// Implements the FFTW 3 single-precision subset the reference calls
// (declared in shim_include/fftw3.h) on top of oracle/cpu_fft.hpp, so the
// unmodified reference CPU sources can be linked and run here.  Semantics
// follow FFTW's documentation: unnormalised transforms, r2c forward
// (sign -1), c2r backward (sign +1), (n0,n1,n2) row-major with n2 halved.
// c2r preserves its input (FFTW may destroy it; the reference never relies
// on either behaviour).  Thread count comes from fftwf_plan_with_nthreads,
// which the reference sets from CLARITY_NP or omp_get_num_procs
// (src/Clarity.cxx:52-58,93-103).
#include <cstdlib>
#include <new>

#include "cpu_fft.hpp"
#include "fftw3.h"

struct fftwf_plan_s {
  int kind;  // 0 = r2c, 1 = c2r
  int n0, n1, n2;
  float *real;
  fftwf_complex *cplx;
};

static int g_nthreads = 1;

extern "C" {

fftwf_plan fftwf_plan_dft_r2c_3d(int n0, int n1, int n2, float *in,
                                 fftwf_complex *out, unsigned) {
  if (n0 <= 0 || n1 <= 0 || n2 <= 0) return nullptr;
  fftwf_plan p = new (std::nothrow) fftwf_plan_s{0, n0, n1, n2, in, out};
  return p;
}

fftwf_plan fftwf_plan_dft_c2r_3d(int n0, int n1, int n2, fftwf_complex *in,
                                 float *out, unsigned) {
  if (n0 <= 0 || n1 <= 0 || n2 <= 0) return nullptr;
  fftwf_plan p = new (std::nothrow) fftwf_plan_s{1, n0, n1, n2, out, in};
  return p;
}

void fftwf_execute(const fftwf_plan p) {
  if (!p) return;
#ifdef _OPENMP
  omp_set_num_threads(g_nthreads > 0 ? g_nthreads : 1);
#endif
  auto *c = reinterpret_cast<std::complex<float> *>(p->cplx);
  if (p->kind == 0)
    oracle::r2c_3d<float>(p->n0, p->n1, p->n2, p->real, c);
  else
    oracle::c2r_3d<float>(p->n0, p->n1, p->n2, c, p->real);
}

void fftwf_destroy_plan(fftwf_plan p) { delete p; }

void *fftwf_malloc(size_t n) {
  void *ptr = nullptr;
  if (posix_memalign(&ptr, 64, n ? n : 64) != 0) return nullptr;
  return ptr;
}

void fftwf_free(void *p) { free(p); }

int fftwf_init_threads(void) { return 1; }

void fftwf_cleanup_threads(void) {}

void fftwf_plan_with_nthreads(int nthreads) {
  g_nthreads = nthreads > 0 ? nthreads : 1;
}

}  // extern "C"
