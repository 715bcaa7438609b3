// clarity_oracle.cpp -- TEST INFRASTRUCTURE ONLY (oracle).
//
// CPU restatement of the reference deconvolution path, used as the parity
// checker for the CUDA library.  Only tests/, __graft_entry__.smoke() and
// bench.py's CPU-baseline leg load it.  Every algorithm is templated on the
// arithmetic type T (float reproduces the reference's FFTW float path; double
// is the FP64 oracle every result's error is stated against) and follows the
// cited reference lines step by step.  FFTs come from cpu_fft.hpp, a
// restatement of FFTW's published transform definitions.
//
// Sum modes for the RL flux rescale (src/MaximumLikelihoodDeconvolve.cxx:73-78):
//   SUM_SERIAL_T  serial accumulation in T, as Clarity_ReduceSum's CPU branch
//                 (src/ComputePrimitives.cxx:61-71)
//   SUM_DOUBLE    accumulation in double, rounded to T once (the parity
//                 target; the CUDA library sums in FP64)
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "cpu_fft.hpp"

namespace {

enum { SUM_SERIAL_T = 0, SUM_DOUBLE = 1 };

struct Dim3 {
  int x, y, z;
  long n() const { return (long)x * y * z; }
};

// src/ImagePadSpatialShift.cxx:32-69: dst[d] = src[(d - shift) mod dstDim]
// when that index lies inside src, else fill.
template <class T, class S>
void pad_shift(T* dst, Dim3 dd, const S* src, Dim3 sd, const int shift[3],
               T fill) {
  for (int dk = 0; dk < dd.z; dk++) {
    int sk = dk - shift[2];
    if (sk < 0) sk += dd.z;
    sk = sk % dd.z;
    bool wk = sk >= 0 && sk < sd.z;
    for (int dj = 0; dj < dd.y; dj++) {
      int sj = dj - shift[1];
      if (sj < 0) sj += dd.y;
      sj = sj % dd.y;
      bool wj = sj >= 0 && sj < sd.y;
      for (int di = 0; di < dd.x; di++) {
        int si = di - shift[0];
        if (si < 0) si += dd.x;
        si = si % dd.x;
        bool wi = si >= 0 && si < sd.x;
        long d = ((long)dk * dd.y + dj) * dd.x + di;
        if (wi && wj && wk)
          dst[d] = (T)src[((long)sk * sd.y + sj) * sd.x + si];
        else
          dst[d] = fill;
      }
    }
  }
}

// src/ImageClip.cxx:30-50: crop from the origin.
template <class T, class D>
void clip(D* dst, Dim3 dd, const T* src, Dim3 sd) {
  for (int k = 0; k < dd.z; k++)
    for (int j = 0; j < dd.y; j++)
      for (int i = 0; i < dd.x; i++)
        dst[((long)k * dd.y + j) * dd.x + i] =
            (D)src[((long)k * sd.y + j) * sd.x + i];
}

template <class T>
struct Work {
  Dim3 img, ker, wd;
  long n, nc;
  std::vector<T> g, h;  // padded image, padded+shifted kernel
  template <class S>
  Work(const S* in, Dim3 id, const S* kernel, Dim3 kd) : img(id), ker(kd) {
    // src/MaximumLikelihoodDeconvolve.cxx:271-292 (same in every algorithm):
    // work = image + kernel; image padded with zero shift, kernel shifted by
    // -kernelDim/2 (truncating division) so its centre sits at the origin.
    wd = Dim3{id.x + kd.x, id.y + kd.y, id.z + kd.z};
    n = wd.n();
    nc = (long)wd.z * wd.y * (wd.x / 2 + 1);
    g.resize(n);
    h.resize(n);
    const int zero[3] = {0, 0, 0};
    const int ks[3] = {-kd.x / 2, -kd.y / 2, -kd.z / 2};
    pad_shift<T, S>(g.data(), wd, in, id, zero, (T)0);
    pad_shift<T, S>(h.data(), wd, kernel, kd, ks, (T)0);
  }
  void r2c(const T* in, oracle::cx<T>* out) const {
    oracle::r2c_3d<T>(wd.z, wd.y, wd.x, in, out);
  }
  void c2r(const oracle::cx<T>* in, T* out) const {
    oracle::c2r_3d<T>(wd.z, wd.y, wd.x, in, out);
  }
};

// src/Convolve.cxx:195-205 / include/internal/Complex.h:95-102:
// out = scale * (a * b), complex multiply without conjugation.
template <class T>
void modulate(long nc, const oracle::cx<T>* a, const oracle::cx<T>* b,
              T scale, oracle::cx<T>* out) {
  for (long i = 0; i < nc; i++) {
    T ar = a[i].real(), ai = a[i].imag(), br = b[i].real(), bi = b[i].imag();
    out[i] = oracle::cx<T>(scale * (ar * br - ai * bi),
                           scale * (ar * bi + ai * br));
  }
}

template <class T>
T inv_n(const Dim3& wd) {
  // src/Convolve.cxx:199: 1.0f / ((float) nz*ny*nx)
  return (T)1 / ((T)wd.z * wd.y * wd.x);
}

// src/Convolve.cxx:118-143: out = C2R(R2C(in) * otf / N)
template <class T>
void convolve_otf(const Work<T>& w, const T* in, const oracle::cx<T>* otf,
                  T* out, std::vector<oracle::cx<T>>& tmp) {
  w.r2c(in, tmp.data());
  modulate<T>(w.nc, tmp.data(), otf, inv_n<T>(w.wd), tmp.data());
  w.c2r(tmp.data(), out);
}

template <class T>
T reduce_sum(const T* a, long n, int mode) {
  if (mode == SUM_SERIAL_T) {
    T s = 0;
    for (long i = 0; i < n; i++) s += a[i];
    return s;
  }
  double s = 0;
  for (long i = 0; i < n; i++) s += (double)a[i];
  return (T)s;
}

// conj(v) in place: the spectrum of the reflected kernel, h(-x), so that a
// product with it is a correlation with h (no reference counterpart: the
// reference never conjugates, src/MaximumLikelihoodDeconvolve.cxx:57,65).
template <class T>
void conjugate(std::vector<oracle::cx<T>>& v) {
  for (auto& c : v) c = oracle::cx<T>(c.real(), -c.imag());
}

// Clarity_Convolve: src/Convolve.cxx:41-115,146-184.  correlate: the
// kernel's spectrum is conjugated first (circular correlation; an opt-in of
// this library with no reference counterpart).
template <class T, class S>
void convolve(const S* in, Dim3 id, const S* kernel, Dim3 kd, S* out,
              T* out_work, bool correlate = false) {
  Work<T> w(in, id, kernel, kd);
  std::vector<oracle::cx<T>> a(w.nc), b(w.nc);
  std::vector<T> o(w.n);
  w.r2c(w.g.data(), a.data());
  w.r2c(w.h.data(), b.data());
  if (correlate) conjugate<T>(b);
  modulate<T>(w.nc, a.data(), b.data(), inv_n<T>(w.wd), a.data());
  w.c2r(a.data(), o.data());
  clip<T, S>(out, id, o.data(), w.wd);
  if (out_work) std::memcpy(out_work, o.data(), sizeof(T) * w.n);
}

// I-divergence of the image against b (a work-box volume) over the image
// region: g ln(g/b) + b - g, 0 ln 0 = 0, terms with g > 0 >= b skipped (the
// definition of oracle_idivergence), in double.
template <class T>
double idiv_image(const Work<T>& w, Dim3 id, const T* b) {
  double acc = 0;
  for (int z = 0; z < id.z; z++)
    for (int y = 0; y < id.y; y++)
      for (int x = 0; x < id.x; x++) {
        const long i = ((long)z * w.wd.y + y) * w.wd.x + x;
        const double a = (double)w.g[i], bb = (double)b[i];
        if (a > 0) {
          if (bb > 0) acc += a * std::log(a / bb) + bb - a;
        } else {
          acc += bb - a;
        }
      }
  return acc;
}

// Richardson-Lucy / ML: src/MaximumLikelihoodDeconvolve.cxx:84-153 with the
// update of :48-81.  The returned estimate is the last iterate; the reference
// leaves the output unwritten when iterations == 0, here the padded input is
// returned (the state RL starts from).
//
// Extensions (no reference counterpart): `start` replaces the image as the
// first estimate (an image-sized volume, zero-padded like the image); `idiv`
// receives, per iteration, the I-divergence of the image against s1 = h * u
// over the image region (the definition of oracle_idivergence, in double).
//
// correlate (no reference counterpart): the second convolution of every
// iteration (:65) uses the conjugated OTF -- a correlation with h, the
// textbook h^T of Richardson-Lucy -- instead of the reference's h.
template <class T, class S>
void rl(const S* in, Dim3 id, const S* kernel, Dim3 kd, S* out, int iters,
        int sum_mode, T* out_work, const S* start = nullptr, double* idiv = nullptr,
        bool correlate = false) {
  Work<T> w(in, id, kernel, kd);
  const long n = w.n;
  std::vector<oracle::cx<T>> otf(w.nc), tmp(w.nc), otf2;
  w.r2c(w.h.data(), otf.data());                      // :98
  if (correlate) {
    otf2 = otf;
    conjugate<T>(otf2);
  }
  const oracle::cx<T>* second = correlate ? otf2.data() : otf.data();
  std::vector<T> u(w.g), s1(n), s2(n);
  if (start) {
    const int zero[3] = {0, 0, 0};
    pad_shift<T, S>(u.data(), w.wd, start, id, zero, (T)0);
  }
  const T energy = reduce_sum<T>(w.g.data(), n, sum_mode);  // :133
  for (int k = 0; k < iters; k++) {
    // :57 s1 = h * u (no conjugate)
    convolve_otf<T>(w, u.data(), otf.data(), s1.data(), tmp);
    if (idiv) idiv[k] = idiv_image(w, id, s1.data());
    // :62 s1 = g / s1 with |s1| < 1e-5 -> 0 (src/ComputePrimitives.cxx:144-148);
    // the comparison is made in double, as fabs(float) < 1e-5 is in C++
    for (long i = 0; i < n; i++)
      s1[i] = ((double)std::fabs(s1[i]) < 1e-5) ? (T)0 : w.g[i] / s1[i];
    // :65 s2 = h * s1
    convolve_otf<T>(w, s1.data(), second, s2.data(), tmp);
    // :69-70 u = u * s2
    for (long i = 0; i < n; i++) u[i] = u[i] * s2[i];
    // :73-78 flux rescale over the whole padded box
    const T ne = reduce_sum<T>(u.data(), n, sum_mode);
    const T scale = energy / ne;
    for (long i = 0; i < n; i++) u[i] = scale * u[i];
  }
  if (idiv) {  // the result's own I-divergence (the start's, without iterations)
    convolve_otf<T>(w, u.data(), otf.data(), s1.data(), tmp);
    idiv[iters] = idiv_image(w, id, s1.data());
  }
  clip<T, S>(out, id, u.data(), w.wd);
  if (out_work) std::memcpy(out_work, u.data(), sizeof(T) * n);
}

// Accelerated Richardson-Lucy (no reference counterpart): vector
// extrapolation of Biggs and Andrews ("Acceleration of iterative image
// restoration algorithms", Applied Optics 36(8):1766-1775, 1997).  Per
// iteration k: y = max(0, x + alpha (x - x_prev)); x_next = RL step at y (the
// update and flux rescale above); g_k = x_next - y; alpha for the next
// iteration = sum(g_k g_{k-1}) / sum(g_{k-1}^2) clamped to [0, 1] (0 until two
// steps exist).  idiv[k] is the I-divergence at y, idiv[iters] that of the
// result.  The extrapolation uses one fused multiply-add, as the GPU does.
template <class T, class S>
void rl_accel(const S* in, Dim3 id, const S* kernel, Dim3 kd, S* out, int iters,
              int sum_mode, double* idiv) {
  Work<T> w(in, id, kernel, kd);
  const long n = w.n;
  std::vector<oracle::cx<T>> otf(w.nc), tmp(w.nc);
  w.r2c(w.h.data(), otf.data());
  std::vector<T> x(w.g), xp(w.g), y(n), s1(n), s2(n), gk(n, (T)0), xn(n);
  const T energy = reduce_sum<T>(w.g.data(), n, sum_mode);
  T alpha = 0;
  for (int k = 0; k < iters; k++) {
    for (long i = 0; i < n; i++) {
      const T v = std::fma(alpha, x[i] - xp[i], x[i]);
      y[i] = v > (T)0 ? v : (T)0;
    }
    convolve_otf<T>(w, y.data(), otf.data(), s1.data(), tmp);
    if (idiv) idiv[k] = idiv_image(w, id, s1.data());
    for (long i = 0; i < n; i++)
      s1[i] = ((double)std::fabs(s1[i]) < 1e-5) ? (T)0 : w.g[i] / s1[i];
    convolve_otf<T>(w, s1.data(), otf.data(), s2.data(), tmp);
    for (long i = 0; i < n; i++) xn[i] = y[i] * s2[i];
    const T ne = reduce_sum<T>(xn.data(), n, sum_mode);
    const T scale = energy / ne;
    double d1 = 0, d2 = 0;
    for (long i = 0; i < n; i++) {
      const T v = scale * xn[i];
      const T g = v - y[i];
      if (k > 0) {
        d1 += (double)g * (double)gk[i];
        d2 += (double)gk[i] * (double)gk[i];
      }
      gk[i] = g;
      xn[i] = v;
    }
    if (k > 0 && d2 > 0) {
      const T a = (T)(d1 / d2);
      alpha = a < (T)0 ? (T)0 : (a > (T)1 ? (T)1 : a);
    } else {
      alpha = 0;
    }
    xp.swap(x);
    x.swap(xn);
  }
  if (idiv && iters > 0) {
    convolve_otf<T>(w, x.data(), otf.data(), s1.data(), tmp);
    idiv[iters] = idiv_image(w, id, s1.data());
  }
  clip<T, S>(out, id, x.data(), w.wd);
}

// Blind ML with the PSF update (no reference counterpart: the reference
// leaves it disabled, src/BlindMaximumLikelihoodDeconvolve.cxx:96).  h starts
// as the padded kernel over its sum (:59); per outer iteration one object step
// o <- o (h * (g / (h * o))) (:63-93), then `sub` PSF steps
// h <- h (o * (g / (h * o))), each renormalised to unit sum.  psf_out (kernel
// grid) receives h through the inverse of the pad/shift.
template <class T, class S>
void blind_psf(const S* in, Dim3 id, const S* kernel, Dim3 kd, S* out, S* psf_out, int iters,
               int sub) {
  Work<T> w(in, id, kernel, kd);
  const long n = w.n;
  std::vector<oracle::cx<T>> Hf(w.nc), Of(w.nc), tmp(w.nc);
  std::vector<T> o(w.g), h(w.h), s1(n), s2(n);
  {
    const T sum = reduce_sum<T>(h.data(), n, SUM_DOUBLE);
    const T inv = (T)1 / sum;
    for (long i = 0; i < n; i++) h[i] = inv * h[i];
  }
  auto step = [&](std::vector<T>& x, const std::vector<oracle::cx<T>>& F) {
    convolve_otf<T>(w, x.data(), F.data(), s1.data(), tmp);
    for (long i = 0; i < n; i++)
      s1[i] = ((double)std::fabs(s1[i]) < 1e-5) ? (T)0 : w.g[i] / s1[i];
    convolve_otf<T>(w, s1.data(), F.data(), s2.data(), tmp);
    for (long i = 0; i < n; i++) x[i] = x[i] * s2[i];
  };
  for (int k = 0; k < iters; k++) {
    w.r2c(h.data(), Hf.data());
    step(o, Hf);
    if (sub > 0) w.r2c(o.data(), Of.data());
    for (int j = 0; j < sub; j++) {
      step(h, Of);
      const T ne = reduce_sum<T>(h.data(), n, SUM_DOUBLE);
      const T scale = (T)1 / ne;
      for (long i = 0; i < n; i++) h[i] = scale * h[i];
    }
  }
  clip<T, S>(out, id, o.data(), w.wd);
  if (psf_out) {
    for (int z = 0; z < kd.z; z++)
      for (int y = 0; y < kd.y; y++)
        for (int x = 0; x < kd.x; x++) {
          const int dx = ((x - kd.x / 2) % w.wd.x + w.wd.x) % w.wd.x;
          const int dy = ((y - kd.y / 2) % w.wd.y + w.wd.y) % w.wd.y;
          const int dz = ((z - kd.z / 2) % w.wd.z + w.wd.z) % w.wd.z;
          psf_out[((long)z * kd.y + y) * kd.x + x] =
              (S)h[((long)dz * w.wd.y + dy) * w.wd.x + dx];
        }
  }
}

// Wiener: src/WienerDeconvolve.cxx:69-122 with the kernel of :48-66.
template <class T, class S>
void wiener(const S* in, Dim3 id, const S* kernel, Dim3 kd, S* out, T eps,
            T* out_work) {
  Work<T> w(in, id, kernel, kd);
  std::vector<oracle::cx<T>> G(w.nc), H(w.nc);
  std::vector<T> o(w.n);
  w.r2c(w.g.data(), G.data());
  w.r2c(w.h.data(), H.data());
  const T scale = inv_n<T>(w.wd);
  for (long i = 0; i < w.nc; i++) {
    T hr = H[i].real(), hi = -H[i].imag();       // conj(H)
    T mag = H[i].real() * H[i].real() + H[i].imag() * H[i].imag();
    T f = (T)1 / (mag + eps);
    hr *= f;
    hi *= f;
    T gr = G[i].real(), gi = G[i].imag();
    G[i] = oracle::cx<T>(scale * (hr * gr - hi * gi),
                         scale * (hr * gi + hi * gr));
  }
  w.c2r(G.data(), o.data());
  clip<T, S>(out, id, o.data(), w.wd);
  if (out_work) std::memcpy(out_work, o.data(), sizeof(T) * w.n);
}

// Sampled Gaussian smoothing kernel for smoothed JVC, as a PSF of the work
// box size: exp(-d^2 / (2 sigma^2)) per axis about the centre n/2 (a delta
// along an axis with sigma <= 0), normalised to unit sum in double, then
// rounded to float.  The reference has no definition to follow
// (src/SmoothedJansenVanCittertDeconvolve.cxx:27-40 writes zeros); the CUDA
// library builds the same kernel.
std::vector<float> gauss_kernel(Dim3 wd, const double sigma[3]) {
  const int n[3] = {wd.x, wd.y, wd.z};
  std::vector<double> ax[3];
  for (int d = 0; d < 3; ++d) {
    ax[d].resize(n[d]);
    const int c = n[d] / 2;
    for (int i = 0; i < n[d]; ++i) {
      const double t = i - c;
      ax[d][i] = sigma[d] > 0 ? std::exp(-t * t / (2.0 * sigma[d] * sigma[d])) : (i == c ? 1.0 : 0.0);
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

// JVC: src/JansenVanCittertDeconvolve.cxx:122-192 with the update of
// :90-119 and A = max(unpadded image)/2 (:128-129, :324).  iterations <= 1
// performs exactly one update (:167-173).  Smoothed JVC (interval > 0):
// after every interval-th update the estimate on the work box is convolved
// with gauss_kernel(sigma) (pad/shift as any PSF, then C2R(R2C(i) G / N)).
template <class T, class S>
void jvc(const S* in, Dim3 id, const S* kernel, Dim3 kd, S* out, int iters,
         T* out_work, int interval = 0, const double* sigma = nullptr) {
  Work<T> w(in, id, kernel, kd);
  const long n = w.n;
  T mx = (T)in[0];
  for (long i = 0; i < id.n(); i++)
    if ((T)in[i] > mx) mx = (T)in[i];
  const T A = (T)0.5 * mx;
  const T invASq = (T)1 / (A * A);
  std::vector<oracle::cx<T>> otf(w.nc), tmp(w.nc);
  w.r2c(w.h.data(), otf.data());
  std::vector<T> i_k(w.g), o(n);
  std::vector<oracle::cx<T>> gotf;
  if (interval > 0) {
    const std::vector<float> gk = gauss_kernel(w.wd, sigma);
    std::vector<T> gpad(n);
    const int sh[3] = {-w.wd.x / 2, -w.wd.y / 2, -w.wd.z / 2};
    pad_shift<T, float>(gpad.data(), w.wd, gk.data(), w.wd, sh, (T)0);
    gotf.resize(w.nc);
    w.r2c(gpad.data(), gotf.data());
  }
  const int total = iters > 1 ? iters : 1;
  for (int k = 0; k < total; k++) {
    convolve_otf<T>(w, i_k.data(), otf.data(), o.data(), tmp);
    for (long j = 0; j < n; j++) {
      T diff = o[j] - A;
      T gamma = (T)1 - ((diff * diff) * invASq);
      T val = i_k[j] + (gamma * (w.g[j] - o[j]));
      if (val < (T)0) val = (T)0;
      i_k[j] = val;
    }
    if (interval > 0 && (k + 1) % interval == 0) {
      convolve_otf<T>(w, i_k.data(), gotf.data(), o.data(), tmp);
      i_k.swap(o);
    }
  }
  clip<T, S>(out, id, i_k.data(), w.wd);
  if (out_work) std::memcpy(out_work, i_k.data(), sizeof(T) * n);
}

// Blind ML, reference CPU semantics: src/BlindMaximumLikelihoodDeconvolve.cxx
// :102-148 with the update of :50-99.  h is renormalised to unit sum at the
// start of every update (:59, Clarity_NormalizeArray) but never updated
// (:96 is disabled); the discarded third convolution (:89-93) has no effect
// on the result and is skipped; there is no flux rescale.
template <class T, class S>
void blind(const S* in, Dim3 id, const S* kernel, Dim3 kd, S* out, int iters,
           int sum_mode, T* out_work) {
  Work<T> w(in, id, kernel, kd);
  const long n = w.n;
  std::vector<oracle::cx<T>> O(w.nc), Hk(w.nc), t1(w.nc);
  std::vector<T> u(w.g), tmp(n);
  const T scale = inv_n<T>(w.wd);
  for (int k = 0; k < iters; k++) {
    // src/ComputePrimitives.cxx:197-209: h = h * (1 / sum h)
    const T sum = reduce_sum<T>(w.h.data(), n, sum_mode);
    const T inv = (T)1 / sum;
    for (long i = 0; i < n; i++) w.h[i] = inv * w.h[i];
    w.r2c(u.data(), O.data());
    w.r2c(w.h.data(), Hk.data());
    modulate<T>(w.nc, O.data(), Hk.data(), scale, t1.data());
    w.c2r(t1.data(), tmp.data());
    for (long i = 0; i < n; i++)
      tmp[i] = ((double)std::fabs(tmp[i]) < 1e-5) ? (T)0 : w.g[i] / tmp[i];
    w.r2c(tmp.data(), t1.data());
    modulate<T>(w.nc, t1.data(), Hk.data(), scale, t1.data());
    w.c2r(t1.data(), tmp.data());
    for (long i = 0; i < n; i++) u[i] = u[i] * tmp[i];
  }
  clip<T, S>(out, id, u.data(), w.wd);
  if (out_work) std::memcpy(out_work, u.data(), sizeof(T) * n);
}

// I-divergence restoration after J. Markham and J.A. Conchello, "Fast
// maximum-likelihood image-restoration algorithms for three-dimensional
// fluorescence microscopy", J. Opt. Soc. Am. A 18(5), 2001 -- the method the
// reference declares (Clarity.h.in:294-319) and leaves a stub
// (src/IDivergenceDeconvolve.cxx: the functional of :33-47, an empty
// gradient).  No reference output exists to pin this restatement to.
//
// Minimises J(s) = sum g ln(g / gh) + gh - g + alpha sum s^2 over the work box
// (g zero-padded, gh = h * s) with s = a^2, by Polak-Ribiere conjugate
// gradients on a:
//   gradient   dJ/da = 2 a (h (x) (1 - g/gh) + 2 alpha a^2), (x) = correlation
//              (the OTF conjugated), g/gh with the RL guard (gh <= 1e-5 -> 0);
//   direction  d = -grad + beta d, beta = max(0, grad'.(grad' - grad) / grad.grad);
//   step       gh(l) = gh + l h*(2 a d) + l^2 h*(d d) exactly, and kNewton
//              Newton steps on dJ/dl from l = 0 (per-voxel terms and sums in
//              double; l >= 0; a step with a non-positive second derivative
//              keeps l); then a += l d, gh = gh(l).
// Starts from a = sqrt(g); returns s = a^2 on the image region.
constexpr int kNewton = 4;

template <class T, class S>
void idiv_cg(const S* in, Dim3 id, const S* kernel, Dim3 kd, S* out, int iters, double alpha) {
  Work<T> w(in, id, kernel, kd);
  const long n = w.n;
  std::vector<oracle::cx<T>> otf(w.nc), otfc(w.nc), tmp(w.nc);
  w.r2c(w.h.data(), otf.data());
  for (long i = 0; i < w.nc; i++) otfc[i] = std::conj(otf[i]);
  std::vector<T> a(n), d(n), gr(n), grn(n), g0(n), p1(n), p2(n), t(n);
  auto ratio = [](double g, double b) { return b > 1e-5 ? g / b : 0.0; };
  auto gradient = [&]() {
    for (long i = 0; i < n; i++) t[i] = (T)(1.0 - ratio(w.g[i], g0[i]));
    convolve_otf<T>(w, t.data(), otfc.data(), t.data(), tmp);
    for (long i = 0; i < n; i++)
      grn[i] = (T)2 * a[i] * (t[i] + (T)(2.0 * alpha) * a[i] * a[i]);
  };
  for (long i = 0; i < n; i++) a[i] = std::sqrt(w.g[i] > 0 ? w.g[i] : (T)0);
  for (long i = 0; i < n; i++) t[i] = a[i] * a[i];
  convolve_otf<T>(w, t.data(), otf.data(), g0.data(), tmp);
  gradient();
  for (long i = 0; i < n; i++) {
    gr[i] = grn[i];
    d[i] = -grn[i];
  }
  for (int k = 0; k < iters; k++) {
    for (long i = 0; i < n; i++) t[i] = (T)2 * a[i] * d[i];
    convolve_otf<T>(w, t.data(), otf.data(), p1.data(), tmp);
    for (long i = 0; i < n; i++) t[i] = d[i] * d[i];
    convolve_otf<T>(w, t.data(), otf.data(), p2.data(), tmp);
    double l = 0;
    for (int m = 0; m < kNewton; m++) {
      double f1 = 0, f2 = 0;
      for (long i = 0; i < n; i++) {
        const double gh = (double)g0[i] + l * (double)p1[i] + l * l * (double)p2[i];
        const double gp = (double)p1[i] + 2.0 * l * (double)p2[i];
        const double r = ratio(w.g[i], gh);
        f1 += (1.0 - r) * gp;
        f2 += (gh > 1e-5 ? r / gh : 0.0) * gp * gp + (1.0 - r) * 2.0 * (double)p2[i];
        const double sl = (double)a[i] + l * (double)d[i], dd = (double)d[i];
        f1 += 4.0 * alpha * sl * sl * sl * dd;
        f2 += 12.0 * alpha * sl * sl * dd * dd;
      }
      if (f2 > 0) {
        l -= f1 / f2;
        if (l < 0) l = 0;
      }
    }
    const T lf = (T)l, l2 = (T)(l * l);
    for (long i = 0; i < n; i++) {
      a[i] = a[i] + lf * d[i];
      g0[i] = g0[i] + lf * p1[i] + l2 * p2[i];
    }
    gradient();
    double num = 0, den = 0;
    for (long i = 0; i < n; i++) {
      num += (double)grn[i] * ((double)grn[i] - (double)gr[i]);
      den += (double)gr[i] * (double)gr[i];
    }
    double beta = den > 0 ? num / den : 0.0;
    if (beta < 0) beta = 0;
    const T bf = (T)beta;
    for (long i = 0; i < n; i++) {
      d[i] = -grn[i] + bf * d[i];
      gr[i] = grn[i];
    }
  }
  for (long i = 0; i < n; i++) t[i] = a[i] * a[i];
  clip<T, S>(out, id, t.data(), w.wd);
}

}  // namespace

// ---------------------------------------------------------------- C ABI ---
// Volumes are x-fastest float arrays; *_f64 variants compute in double but
// take and return float volumes (the padded work-box result, when requested
// through out_work, is returned in the computing precision).
extern "C" {

#define ORACLE_DIMS                                                   \
  Dim3 id{ix, iy, iz};                                                \
  Dim3 kd{kx, ky, kz}

void oracle_convolve_f32(const float* in, int ix, int iy, int iz,
                         const float* k, int kx, int ky, int kz, float* out,
                         float* work) {
  ORACLE_DIMS;
  convolve<float, float>(in, id, k, kd, out, work);
}
void oracle_convolve_f64(const float* in, int ix, int iy, int iz,
                         const float* k, int kx, int ky, int kz, float* out,
                         double* work) {
  ORACLE_DIMS;
  convolve<double, float>(in, id, k, kd, out, work);
}
void oracle_correlate_f32(const float* in, int ix, int iy, int iz,
                          const float* k, int kx, int ky, int kz, float* out) {
  ORACLE_DIMS;
  convolve<float, float>(in, id, k, kd, out, (float*)nullptr, true);
}
void oracle_correlate_f64(const float* in, int ix, int iy, int iz,
                          const float* k, int kx, int ky, int kz, float* out) {
  ORACLE_DIMS;
  convolve<double, float>(in, id, k, kd, out, (double*)nullptr, true);
}
void oracle_rl_corr_f32(const float* in, int ix, int iy, int iz, const float* k,
                        int kx, int ky, int kz, float* out, int iters) {
  ORACLE_DIMS;
  rl<float, float>(in, id, k, kd, out, iters, SUM_DOUBLE, (float*)nullptr, nullptr, nullptr,
                   true);
}
void oracle_rl_corr_f64(const float* in, int ix, int iy, int iz, const float* k,
                        int kx, int ky, int kz, float* out, int iters) {
  ORACLE_DIMS;
  rl<double, float>(in, id, k, kd, out, iters, SUM_DOUBLE, (double*)nullptr, nullptr, nullptr,
                    true);
}
void oracle_rl_f32(const float* in, int ix, int iy, int iz, const float* k,
                   int kx, int ky, int kz, float* out, int iters,
                   int sum_mode, float* work) {
  ORACLE_DIMS;
  rl<float, float>(in, id, k, kd, out, iters, sum_mode, work);
}
void oracle_rl_f64(const float* in, int ix, int iy, int iz, const float* k,
                   int kx, int ky, int kz, float* out, int iters,
                   double* work) {
  ORACLE_DIMS;
  rl<double, float>(in, id, k, kd, out, iters, SUM_DOUBLE, work);
}
void oracle_rl_ex_f32(const float* in, int ix, int iy, int iz, const float* k,
                      int kx, int ky, int kz, float* out, int iters, int sum_mode,
                      const float* start, double* idiv, float* work) {
  ORACLE_DIMS;
  rl<float, float>(in, id, k, kd, out, iters, sum_mode, work, start, idiv);
}
void oracle_rl_ex_f64(const float* in, int ix, int iy, int iz, const float* k,
                      int kx, int ky, int kz, float* out, int iters,
                      const float* start, double* idiv, double* work) {
  ORACLE_DIMS;
  rl<double, float>(in, id, k, kd, out, iters, SUM_DOUBLE, work, start, idiv);
}
void oracle_rl_accel_f32(const float* in, int ix, int iy, int iz, const float* k,
                         int kx, int ky, int kz, float* out, int iters, int sum_mode,
                         double* idiv) {
  ORACLE_DIMS;
  rl_accel<float, float>(in, id, k, kd, out, iters, sum_mode, idiv);
}
void oracle_rl_accel_f64(const float* in, int ix, int iy, int iz, const float* k,
                         int kx, int ky, int kz, float* out, int iters, double* idiv) {
  ORACLE_DIMS;
  rl_accel<double, float>(in, id, k, kd, out, iters, SUM_DOUBLE, idiv);
}
void oracle_blind_psf_f32(const float* in, int ix, int iy, int iz, const float* k, int kx,
                          int ky, int kz, float* out, float* psf_out, int iters, int sub) {
  ORACLE_DIMS;
  blind_psf<float, float>(in, id, k, kd, out, psf_out, iters, sub);
}
void oracle_blind_psf_f64(const float* in, int ix, int iy, int iz, const float* k, int kx,
                          int ky, int kz, float* out, float* psf_out, int iters, int sub) {
  ORACLE_DIMS;
  blind_psf<double, float>(in, id, k, kd, out, psf_out, iters, sub);
}
void oracle_wiener_f32(const float* in, int ix, int iy, int iz,
                       const float* k, int kx, int ky, int kz, float* out,
                       float eps, float* work) {
  ORACLE_DIMS;
  wiener<float, float>(in, id, k, kd, out, eps, work);
}
void oracle_wiener_f64(const float* in, int ix, int iy, int iz,
                       const float* k, int kx, int ky, int kz, float* out,
                       double eps, double* work) {
  ORACLE_DIMS;
  wiener<double, float>(in, id, k, kd, out, eps, work);
}
void oracle_jvc_f32(const float* in, int ix, int iy, int iz, const float* k,
                    int kx, int ky, int kz, float* out, int iters,
                    float* work) {
  ORACLE_DIMS;
  jvc<float, float>(in, id, k, kd, out, iters, work);
}
void oracle_jvc_f64(const float* in, int ix, int iy, int iz, const float* k,
                    int kx, int ky, int kz, float* out, int iters,
                    double* work) {
  ORACLE_DIMS;
  jvc<double, float>(in, id, k, kd, out, iters, work);
}
void oracle_sjvc_f32(const float* in, int ix, int iy, int iz, const float* k,
                     int kx, int ky, int kz, float* out, int iters, int interval,
                     double sx, double sy, double sz, float* work) {
  ORACLE_DIMS;
  const double sg[3] = {sx, sy, sz};
  jvc<float, float>(in, id, k, kd, out, iters, work, interval, sg);
}
void oracle_sjvc_f64(const float* in, int ix, int iy, int iz, const float* k,
                     int kx, int ky, int kz, float* out, int iters, int interval,
                     double sx, double sy, double sz, double* work) {
  ORACLE_DIMS;
  const double sg[3] = {sx, sy, sz};
  jvc<double, float>(in, id, k, kd, out, iters, work, interval, sg);
}
void oracle_blind_f32(const float* in, int ix, int iy, int iz,
                      const float* k, int kx, int ky, int kz, float* out,
                      int iters, int sum_mode, float* work) {
  ORACLE_DIMS;
  blind<float, float>(in, id, k, kd, out, iters, sum_mode, work);
}
void oracle_blind_f64(const float* in, int ix, int iy, int iz,
                      const float* k, int kx, int ky, int kz, float* out,
                      int iters, double* work) {
  ORACLE_DIMS;
  blind<double, float>(in, id, k, kd, out, iters, SUM_DOUBLE, work);
}
void oracle_idiv_cg_f32(const float* in, int ix, int iy, int iz, const float* k, int kx,
                        int ky, int kz, float* out, int iters, double alpha) {
  ORACLE_DIMS;
  idiv_cg<float, float>(in, id, k, kd, out, iters, alpha);
}
void oracle_idiv_cg_f64(const float* in, int ix, int iy, int iz, const float* k, int kx,
                        int ky, int kz, float* out, int iters, double alpha) {
  ORACLE_DIMS;
  idiv_cg<double, float>(in, id, k, kd, out, iters, alpha);
}

// I-divergence of src/IDivergenceDeconvolve.cxx:33-47 with alpha = 0, in
// double: sum over voxels with g > 0 of g ln(g / ghat) + ghat - g, plus ghat
// where g == 0 (0 ln 0 = 0).  Voxels with ghat <= 0 and g > 0 are skipped
// and counted in *skipped.
double oracle_idivergence(const float* g, const float* ghat, long n,
                          long* skipped) {
  double s = 0;
  long sk = 0;
  for (long i = 0; i < n; i++) {
    const double a = g[i], b = ghat[i];
    if (a > 0) {
      if (b <= 0) { sk++; continue; }
      s += a * std::log(a / b) + b - a;
    } else {
      s += b - a;
    }
  }
  if (skipped) *skipped = sk;
  return s;
}

// Pad/shift and clip exactly as the reference public utilities.
void oracle_pad_shift(float* dst, int dx, int dy, int dz, const float* src,
                      int sx, int sy, int sz, const int shift[3], float fill) {
  pad_shift<float, float>(dst, Dim3{dx, dy, dz}, src, Dim3{sx, sy, sz}, shift,
                          fill);
}

// Raw 3-D transforms (FFTW layout) for checking the FFT restatement.
void oracle_r2c_3d_f32(int nz, int ny, int nx, const float* in, float* out) {
  oracle::r2c_3d<float>(nz, ny, nx, in,
                        reinterpret_cast<std::complex<float>*>(out));
}
void oracle_c2r_3d_f32(int nz, int ny, int nx, const float* in, float* out) {
  oracle::c2r_3d<float>(nz, ny, nx,
                        reinterpret_cast<const std::complex<float>*>(in), out);
}
void oracle_r2c_3d_f64(int nz, int ny, int nx, const double* in, double* out) {
  oracle::r2c_3d<double>(nz, ny, nx, in,
                         reinterpret_cast<std::complex<double>*>(out));
}
void oracle_c2r_3d_f64(int nz, int ny, int nx, const double* in, double* out) {
  oracle::c2r_3d<double>(nz, ny, nx,
                         reinterpret_cast<const std::complex<double>*>(in),
                         out);
}

void oracle_set_threads(int n) {
#ifdef _OPENMP
  omp_set_num_threads(n > 0 ? n : 1);
#endif
}

}  // extern "C"
