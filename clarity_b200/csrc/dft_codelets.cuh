// dft_codelets.cuh -- register-resident DFT codelets for sm_100a.
//
// dft<N, DIR>(v) replaces v[0..N) (float2, natural order) with its
// unnormalised DFT, X[k] = sum_t v[t] exp(DIR * 2 pi i t k / N), natural
// order out.  DIR = -1 is the forward transform (the sign FFTW uses for r2c,
// src/FFT.cxx:80), DIR = +1 the backward one.  Every index is a compile-time
// constant (static_for), so the whole codelet lives in registers and every
// twiddle is an immediate operand; trivial twiddles (1, -1, +-i, the
// eighth roots) are special-cased.
//
// Composite N are split Cooley-Tukey style (N = A*B, A = 4 when 4 | N, else
// the smallest prime factor); odd primes use the direct symmetric form that
// pairs t with N - t (about N^2 real multiply-adds).
#pragma once
#include "launch_macro.cuh"

#include <type_traits>
#include <utility>

namespace clarity {

// ------------------------------------------------------------ compile time
template <int I>
using ic = std::integral_constant<int, I>;

template <class F, int... I>
__device__ __forceinline__ void static_for_impl(F&& f,
                                                std::integer_sequence<int, I...>) {
  (f(ic<I>{}), ...);
}
template <int N, class F>
__device__ __forceinline__ void static_for(F&& f) {
  static_for_impl(std::forward<F>(f), std::make_integer_sequence<int, N>{});
}

// cos and sin of 2*pi*k/n at compile time, from the Taylor series on the
// first octant (octant symmetry reduces every angle to [0, pi/4]).  Used only
// for the fixed twiddles inside the codelets.
constexpr double kPi = 3.14159265358979323846264338327950288;

constexpr double taylor_sin(double x) {
  double term = x, sum = x;
  for (int i = 1; i < 30; ++i) {
    term *= -x * x / ((2.0 * i) * (2.0 * i + 1.0));
    sum += term;
  }
  return sum;
}
constexpr double taylor_cos(double x) {
  double term = 1.0, sum = 1.0;
  for (int i = 1; i < 30; ++i) {
    term *= -x * x / ((2.0 * i - 1.0) * (2.0 * i));
    sum += term;
  }
  return sum;
}
// returns {cos, sin} of 2 pi k / n
struct cs_pair {
  double c, s;
};
constexpr cs_pair root_cs(long k, long n) {
  k %= n;
  if (k < 0) k += n;
  // angle = 2 pi k / n ; work with 8k/n in units of octants
  const long k8 = 8 * k;
  const long oct = k8 / n;  // 0..7
  // angle within the octant, measured in radians
  const double frac = (double)(k8 - oct * n) / (double)n;  // [0,1)
  const double a = frac * kPi / 4.0;
  const double ca = taylor_cos(a), sa = taylor_sin(a);
  const double cb = taylor_cos(kPi / 4.0 - a), sb = taylor_sin(kPi / 4.0 - a);
  switch (oct) {
    case 0: return {ca, sa};
    case 1: return {sb, cb};
    case 2: return {-sa, ca};
    case 3: return {-cb, sb};
    case 4: return {-ca, -sa};
    case 5: return {-sb, -cb};
    case 6: return {sa, -ca};
    default: return {cb, -sb};
  }
}

// ------------------------------------------------------------ complex ops
// Complex add and subtract use sm_100's paired FP32 add (one FADD2 per complex
// add instead of two FADDs; each lane rounds exactly as a scalar add), unless
// CLARITY_NO_F32X2 is defined or the code is compiled for the host.
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000 && !defined(CLARITY_NO_F32X2)
#define CLARITY_F32X2 1
#endif
__device__ __forceinline__ float2 cadd(float2 a, float2 b) {
#ifdef CLARITY_F32X2
  return __fadd2_rn(a, b);
#else
  return make_float2(a.x + b.x, a.y + b.y);
#endif
}
__device__ __forceinline__ float2 csub(float2 a, float2 b) {
#ifdef CLARITY_F32X2
  return __fadd2_rn(a, make_float2(-b.x, -b.y));
#else
  return make_float2(a.x - b.x, a.y - b.y);
#endif
}
// a + DIR*i*b, in scalar adds (the lane swap would cost moves in paired form)
template <int DIR>
__device__ __forceinline__ float2 cadd_diri(float2 a, float2 b) {
  if constexpr (DIR < 0)
    return make_float2(a.x + b.y, a.y - b.x);
  else
    return make_float2(a.x - b.y, a.y + b.x);
}
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {
  return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__device__ __forceinline__ float2 conjf2(float2 a) { return make_float2(a.x, -a.y); }
__device__ __forceinline__ float2 cscale(float2 a, float s) {
  return make_float2(a.x * s, a.y * s);
}
// multiply by DIR*i  (DIR = -1: -i, DIR = +1: +i)
template <int DIR>
__device__ __forceinline__ float2 mul_diri(float2 a) {
  if constexpr (DIR < 0)
    return make_float2(a.y, -a.x);
  else
    return make_float2(-a.y, a.x);
}

// v * exp(DIR * 2 pi i K / N), K and N compile time.
template <int K, int N, int DIR>
__device__ __forceinline__ float2 twc(float2 v) {
  constexpr int k = ((K % N) + N) % N;
  if constexpr (k == 0) {
    return v;
  } else if constexpr (2 * k == N) {
    return make_float2(-v.x, -v.y);
  } else if constexpr (4 * k == N) {
    return mul_diri<DIR>(v);
  } else if constexpr (4 * k == 3 * N) {
    return mul_diri<-DIR>(v);
  } else if constexpr (8 * k == N || 8 * k == 3 * N || 8 * k == 5 * N ||
                       8 * k == 7 * N) {
    constexpr float h = 0.70710678118654752440f;
    constexpr cs_pair r = root_cs(k, N);
    constexpr float c = r.c > 0 ? h : -h;
    constexpr float s = (r.s > 0 ? h : -h) * (float)DIR;
    // (v.x + i v.y)(c + i s)
    return make_float2(c * v.x - s * v.y, c * v.y + s * v.x);
  } else {
    constexpr cs_pair r = root_cs(k, N);
    constexpr float c = (float)r.c;
    constexpr float s = (float)(r.s * DIR);
    return make_float2(c * v.x - s * v.y, c * v.y + s * v.x);
  }
}

// ------------------------------------------------------------ factor helper
constexpr int first_split(int n) {
  if (n % 4 == 0 && n > 4) return 4;
  for (int p = 2; p * p <= n; ++p)
    if (n % p == 0) return p;
  return n;  // prime
}

template <int N, int DIR>
struct DFT;

template <int DIR>
struct DFT<1, DIR> {
  __device__ __forceinline__ static void run(float2*) {}
};

template <int DIR>
struct DFT<2, DIR> {
  __device__ __forceinline__ static void run(float2* v) {
    float2 a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  }
};

template <int DIR>
struct DFT<3, DIR> {
  __device__ __forceinline__ static void run(float2* v) {
    constexpr float c = -0.5f;
    constexpr float sn = (float)(DIR * 0.86602540378443864676);
    float2 a0 = v[0], s = cadd(v[1], v[2]), d = csub(v[1], v[2]);
    float2 t = make_float2(a0.x + c * s.x, a0.y + c * s.y);
    float2 jd = make_float2(-sn * d.y, sn * d.x);
    v[0] = cadd(a0, s);
    v[1] = make_float2(t.x + jd.x, t.y + jd.y);
    v[2] = make_float2(t.x - jd.x, t.y - jd.y);
  }
};

template <int DIR>
struct DFT<4, DIR> {
  __device__ __forceinline__ static void run(float2* v) {
    float2 s02 = cadd(v[0], v[2]), d02 = csub(v[0], v[2]);
    float2 s13 = cadd(v[1], v[3]), d13 = csub(v[1], v[3]);
    v[0] = cadd(s02, s13);
    v[1] = cadd_diri<DIR>(d02, d13);
    v[2] = csub(s02, s13);
    v[3] = cadd_diri<-DIR>(d02, d13);
  }
};

// Odd prime N >= 5: symmetric direct form.
template <int N, int DIR>
struct DFTPrime {
  __device__ __forceinline__ static void run(float2* v) {
    constexpr int H = (N - 1) / 2;
    float2 a[H + 1], b[H + 1];
    float2 x0 = v[0];
    float2 X0 = x0;
    static_for<H>([&](auto ti) {
      constexpr int t = decltype(ti)::value + 1;
      a[t] = cadd(v[t], v[N - t]);
      b[t] = csub(v[t], v[N - t]);
      X0 = cadd(X0, a[t]);
    });
    float2 out[N];
    out[0] = X0;
    static_for<H>([&](auto ki) {
      constexpr int k = decltype(ki)::value + 1;
      float2 C = x0, S = make_float2(0.f, 0.f);
      static_for<H>([&](auto ti) {
        constexpr int t = decltype(ti)::value + 1;
        constexpr cs_pair r = root_cs((long)t * k, N);
        constexpr float c = (float)r.c;
        constexpr float s = (float)r.s;
        C.x += c * a[t].x;
        C.y += c * a[t].y;
        S.x += s * b[t].x;
        S.y += s * b[t].y;
      });
      // X[k] = C + DIR*i*S ; X[N-k] = C - DIR*i*S
      out[k] = cadd_diri<DIR>(C, S);
      out[N - k] = cadd_diri<-DIR>(C, S);
    });
    static_for<N>([&](auto ki) {
      constexpr int k = decltype(ki)::value;
      v[k] = out[k];
    });
  }
};

// Composite N = A * B: A-point DFTs with stride B, twiddles, B-point DFTs.
template <int N, int DIR>
struct DFTSplit {
  static constexpr int A = first_split(N);
  static constexpr int B = N / A;
  __device__ __forceinline__ static void run(float2* v) {
    float2 u[N];
    static_for<B>([&](auto ii) {
      constexpr int i = decltype(ii)::value;
      float2 t[A];
      static_for<A>([&](auto ai) {
        constexpr int a = decltype(ai)::value;
        t[a] = v[i + B * a];
      });
      DFT<A, DIR>::run(t);
      static_for<A>([&](auto ki) {
        constexpr int k = decltype(ki)::value;
        u[i + B * k] = twc<i * k, N, DIR>(t[k]);
      });
    });
    static_for<A>([&](auto ki) {
      constexpr int k = decltype(ki)::value;
      float2 s[B];
      static_for<B>([&](auto ii) {
        constexpr int i = decltype(ii)::value;
        s[i] = u[B * k + i];
      });
      DFT<B, DIR>::run(s);
      static_for<B>([&](auto ji) {
        constexpr int j = decltype(ji)::value;
        v[k + A * j] = s[j];
      });
    });
  }
};

constexpr bool is_prime(int n) {
  if (n < 2) return false;
  for (int p = 2; p * p <= n; ++p)
    if (n % p == 0) return false;
  return true;
}

template <int N, int DIR>
struct DFT {
  __device__ __forceinline__ static void run(float2* v) {
    if constexpr (is_prime(N))
      DFTPrime<N, DIR>::run(v);
    else
      DFTSplit<N, DIR>::run(v);
  }
};

template <int N, int DIR>
__device__ __forceinline__ void dft(float2* v) {
  DFT<N, DIR>::run(v);
}

// Radices a runtime plan may use for one register pass.  Every length the
// planner accepts is a product of these.
#define CLARITY_FOR_EACH_RADIX(X) \
  X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13) X(16) X(17) X(19)

constexpr int kMaxRadix = 19;

}  // namespace clarity
