// cpu_fft.hpp -- TEST INFRASTRUCTURE ONLY (oracle).  Nothing in the product
// library links this file; tests, smoke() and bench.py's CPU-baseline leg use
// it through the oracle shared libraries.
//
// A from-scratch CPU implementation of the transforms the reference obtains
// from FFTW 3 (single precision, threads; not vendored, version not pinned by
// the reference: HOWTO-Build-Clarity.txt:5, CMake/FindFFTW.cmake:16,24).
// FFTW's published definition is restated here:
//   forward  X[k] = sum_j x[j] exp(-2 pi i j k / n)   (unnormalised)
//   backward x[j] = sum_k X[k] exp(+2 pi i j k / n)   (unnormalised)
// 3-D real transforms use FFTW's row-major convention with the LAST
// dimension halved: r2c of an (n0,n1,n2) real array gives an
// (n0,n1,n2/2+1) complex array.  The reference passes (nz,ny,nx)
// (src/FFT.cxx:80,131) so x is the halved axis.  For c2r the imaginary parts
// of the self-conjugate bins of the last axis are ignored, as in FFTW's
// rdft2 c2r (complex inverse over the leading axes, then 1-D c2r).
//
// Algorithm: recursive mixed-radix decimation in time (Cooley-Tukey) with
// specialised radix-2/3/4/5 butterflies and a generic odd-prime butterfly;
// twiddles are computed in double and rounded to T.  Even-length real
// transforms use the half-length complex transform plus the standard
// even/odd split.
#ifndef CLARITY_ORACLE_CPU_FFT_HPP_
#define CLARITY_ORACLE_CPU_FFT_HPP_

#include <cmath>
#include <complex>
#include <cstddef>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace oracle {

template <class T>
using cx = std::complex<T>;

// exp(sign * 2 pi i * k / n) computed in double precision.
inline std::complex<double> unit_root(long k, long n, int sign) {
  k %= n;
  if (k < 0) k += n;
  // reduce to the first octant for accuracy
  const double a = 2.0 * M_PI * (double)k / (double)n;
  return std::complex<double>(std::cos(a), sign * std::sin(a));
}

template <class T>
class Plan1D {
 public:
  Plan1D() : n_(0), sign_(-1) {}
  Plan1D(int n, int sign) { init(n, sign); }

  void init(int n, int sign) {
    n_ = n;
    sign_ = sign;
    factors_.clear();
    int m = n;
    while (m % 4 == 0) { factors_.push_back(4); m /= 4; }
    while (m % 2 == 0 && m > 1) { factors_.push_back(2); m /= 2; }
    for (int p = 3; m > 1; p += 2) {
      while (m % p == 0) { factors_.push_back(p); m /= p; }
      if ((long)p * p > m && m > 1) { factors_.push_back(m); m = 1; }
    }
    if (n == 1) factors_.clear();
    tw_.resize(n);
    for (int k = 0; k < n; ++k) {
      std::complex<double> w = unit_root(k, n, sign);
      tw_[k] = cx<T>((T)w.real(), (T)w.imag());
    }
  }

  int size() const { return n_; }

  // out = DFT(in); in is read with stride istride.  out must not alias in.
  void exec(const cx<T>* in, long istride, cx<T>* out) const {
    if (n_ == 1) { out[0] = in[0]; return; }
    rec(in, istride, out, n_, 1, 0);
  }

 private:
  // Transform of length len of in[0], in[s], ... into out[0..len).
  // fstride = n_/len selects the twiddles of this level.
  void rec(const cx<T>* in, long s, cx<T>* out, int len, long fstride,
           size_t fi) const {
    const int p = factors_[fi];
    const int m = len / p;
    if (m == 1) {
      for (int q = 0; q < p; ++q) out[q] = in[(long)q * s];
    } else {
      for (int q = 0; q < p; ++q)
        rec(in + (long)q * s, s * p, out + (long)q * m, m, fstride * p, fi + 1);
    }
    butterfly(out, m, p, fstride);
  }

  // Combine p sub-transforms of length m stored at out[q*m + k].
  void butterfly(cx<T>* out, int m, int p, long fstride) const {
    const cx<T>* tw = tw_.data();
    if (p == 2) {
      for (int k = 0; k < m; ++k) {
        cx<T> a = out[k];
        cx<T> b = out[k + m] * tw[k * fstride];
        out[k] = a + b;
        out[k + m] = a - b;
      }
    } else if (p == 4) {
      for (int k = 0; k < m; ++k) {
        cx<T> a0 = out[k];
        cx<T> a1 = out[k + m] * tw[k * fstride];
        cx<T> a2 = out[k + 2 * m] * tw[2 * k * fstride];
        cx<T> a3 = out[k + 3 * m] * tw[3 * k * fstride];
        cx<T> s02 = a0 + a2, d02 = a0 - a2;
        cx<T> s13 = a1 + a3, d13 = a1 - a3;
        // multiply d13 by sign*i
        cx<T> jd13 = (sign_ < 0) ? cx<T>(d13.imag(), -d13.real())
                                 : cx<T>(-d13.imag(), d13.real());
        out[k] = s02 + s13;
        out[k + m] = d02 + jd13;
        out[k + 2 * m] = s02 - s13;
        out[k + 3 * m] = d02 - jd13;
      }
    } else if (p == 3) {
      const T c = (T)-0.5;
      const T sn = (T)(sign_ * std::sqrt(3.0) / 2.0);
      for (int k = 0; k < m; ++k) {
        cx<T> a0 = out[k];
        cx<T> a1 = out[k + m] * tw[k * fstride];
        cx<T> a2 = out[k + 2 * m] * tw[2 * k * fstride];
        cx<T> s = a1 + a2, d = a1 - a2;
        cx<T> t = a0 + c * s;
        cx<T> jd(-sn * d.imag(), sn * d.real());
        out[k] = a0 + s;
        out[k + m] = t + jd;
        out[k + 2 * m] = t - jd;
      }
    } else {
      // generic radix p: direct DFT of the p twiddled inputs
      std::vector<cx<T>> a(p);
      for (int k = 0; k < m; ++k) {
        for (int q = 0; q < p; ++q)
          a[q] = out[k + q * m] * tw[((long)q * k * fstride) % n_];
        for (int r = 0; r < p; ++r) {
          cx<T> acc = a[0];
          for (int q = 1; q < p; ++q) {
            long e = ((long)q * r % p) * (long)(n_ / p);
            acc += a[q] * tw[e % n_];
          }
          out[k + r * m] = acc;
        }
      }
    }
  }

  int n_;
  int sign_;
  std::vector<int> factors_;
  std::vector<cx<T>> tw_;
};

// 1-D real-to-half-complex transform of length n (forward, sign -1), output
// n/2+1 bins.  Even n uses the half-length complex transform.
template <class T>
class RealPlan {
 public:
  explicit RealPlan(int n) : n_(n) {
    if (n % 2 == 0 && n >= 2) {
      half_.init(n / 2, -1);
      ihalf_.init(n / 2, +1);
      w_.resize(n / 2 + 1);
      for (int k = 0; k <= n / 2; ++k) {
        std::complex<double> w = unit_root(k, n, -1);
        w_[k] = cx<T>((T)w.real(), (T)w.imag());
      }
    } else {
      full_.init(n, -1);
      ifull_.init(n, +1);
    }
  }

  // r2c: in (n reals) -> out (n/2+1 complex).  work >= n complex.
  void forward(const T* in, cx<T>* out, cx<T>* work) const {
    const int n = n_;
    if (n % 2 == 0) {
      const int m = n / 2;
      cx<T>* z = work;
      cx<T>* Z = work + m;
      for (int j = 0; j < m; ++j) z[j] = cx<T>(in[2 * j], in[2 * j + 1]);
      half_.exec(z, 1, Z);
      out[0] = cx<T>(Z[0].real() + Z[0].imag(), 0);
      out[m] = cx<T>(Z[0].real() - Z[0].imag(), 0);
      for (int k = 1; k < m; ++k) {
        cx<T> a = Z[k], b = std::conj(Z[m - k]);
        cx<T> e = (a + b) * (T)0.5;
        cx<T> o = (a - b) * cx<T>(0, (T)-0.5);
        out[k] = e + w_[k] * o;
      }
    } else {
      cx<T>* z = work;
      cx<T>* Z = work + n;
      for (int j = 0; j < n; ++j) z[j] = cx<T>(in[j], 0);
      full_.exec(z, 1, Z);
      for (int k = 0; k <= n / 2; ++k) out[k] = Z[k];
    }
  }

  // c2r: in (n/2+1 complex, Hermitian half) -> out (n reals), unnormalised.
  // Imaginary parts of self-conjugate bins are ignored.  work >= 2n complex.
  void backward(const cx<T>* in, T* out, cx<T>* work) const {
    const int n = n_;
    if (n % 2 == 0) {
      const int m = n / 2;
      cx<T>* Z = work;
      cx<T>* z = work + m;
      const T x0 = in[0].real(), xm = in[m].real();
      Z[0] = cx<T>(x0 + xm, x0 - xm);
      for (int k = 1; k < m; ++k) {
        cx<T> a = in[k], b = std::conj(in[m - k]);
        cx<T> e = a + b;
        cx<T> o = (a - b) * std::conj(w_[k]);
        Z[k] = e + cx<T>(-o.imag(), o.real());
      }
      ihalf_.exec(Z, 1, z);
      for (int j = 0; j < m; ++j) {
        out[2 * j] = z[j].real();
        out[2 * j + 1] = z[j].imag();
      }
    } else {
      cx<T>* Z = work;
      cx<T>* z = work + n;
      Z[0] = cx<T>(in[0].real(), 0);
      for (int k = 1; k <= n / 2; ++k) {
        Z[k] = in[k];
        Z[n - k] = std::conj(in[k]);
      }
      ifull_.exec(Z, 1, z);
      for (int j = 0; j < n; ++j) out[j] = z[j].real();
    }
  }

 private:
  int n_;
  Plan1D<T> half_, ihalf_, full_, ifull_;
  std::vector<cx<T>> w_;
};

// Transform every line along one axis of a complex (nz, ny, nh) array.
// axis 1 = y (stride nh), axis 0 = z (stride ny*nh).
template <class T>
void complex_axis(cx<T>* a, int nz, int ny, int nh, int axis, int sign) {
  const int n = (axis == 1) ? ny : nz;
  if (n == 1) return;
  Plan1D<T> plan(n, sign);
  const long stride = (axis == 1) ? nh : (long)ny * nh;
  const long lines = (long)nz * nh * ny / n;
#pragma omp parallel
  {
    std::vector<cx<T>> buf(n), res(n);
#pragma omp for schedule(static)
    for (long l = 0; l < lines; ++l) {
      long base;
      if (axis == 1) {
        const long z = l / nh, x = l % nh;
        base = z * (long)ny * nh + x;
      } else {
        base = l;  // l in [0, ny*nh)
      }
      for (int j = 0; j < n; ++j) buf[j] = a[base + j * stride];
      plan.exec(buf.data(), 1, res.data());
      for (int j = 0; j < n; ++j) a[base + j * stride] = res[j];
    }
  }
}

// 3-D r2c: real (nz,ny,nx) -> complex (nz,ny,nx/2+1), unnormalised.
template <class T>
void r2c_3d(int nz, int ny, int nx, const T* in, cx<T>* out) {
  const int nh = nx / 2 + 1;
  RealPlan<T> rp(nx);
  const long rows = (long)nz * ny;
#pragma omp parallel
  {
    std::vector<cx<T>> work(2 * (size_t)nx + 2);
#pragma omp for schedule(static)
    for (long r = 0; r < rows; ++r)
      rp.forward(in + r * nx, out + r * nh, work.data());
  }
  complex_axis<T>(out, nz, ny, nh, 1, -1);
  complex_axis<T>(out, nz, ny, nh, 0, -1);
}

// 3-D c2r: complex (nz,ny,nx/2+1) -> real (nz,ny,nx), unnormalised.  The
// input is preserved (a copy is transformed).
template <class T>
void c2r_3d(int nz, int ny, int nx, const cx<T>* in, T* out) {
  const int nh = nx / 2 + 1;
  const size_t count = (size_t)nz * ny * nh;
  std::vector<cx<T>> tmp(in, in + count);
  complex_axis<T>(tmp.data(), nz, ny, nh, 0, +1);
  complex_axis<T>(tmp.data(), nz, ny, nh, 1, +1);
  RealPlan<T> rp(nx);
  const long rows = (long)nz * ny;
#pragma omp parallel
  {
    std::vector<cx<T>> work(2 * (size_t)nx + 2);
#pragma omp for schedule(static)
    for (long r = 0; r < rows; ++r)
      rp.backward(tmp.data() + r * nh, out + r * nx, work.data());
  }
}

}  // namespace oracle

#endif  // CLARITY_ORACLE_CPU_FFT_HPP_
