// passes.cuh -- the fused FFT pass kernels (XY forward, Z, XY inverse and
// XY inverse+forward), templated on the operation fused into them.
//
// Reference counterparts: the 3-D R2C/C2R of src/FFT.cxx:46-146 (cuFFT or
// FFTW), the spectral multiply of src/ModulateGPU.cu:63-93 and
// src/WienerDeconvolveGPU.cu:34-73, and the point-wise kernels of
// src/ComputePrimitivesGPU.cu:148-239 and src/JansenVanCittertDeconvolveGPU.cu
// :38-75, which here become prologues and epilogues of the FFT passes.
#pragma once
#include "launch_macro.cuh"

#include "dft_codelets.cuh"
#include "plan.hpp"

namespace clarity {

// ------------------------------------------------------------------------
// Index arithmetic by runtime divisors.  A pass's work items are numbered
// f = threadIdx.x + k*blockDim.x and split into (line, block, i) by the
// plan's extents; an integer division by a runtime value costs a long
// instruction sequence per item.  DivR keeps d and 1/d (one float division
// per pass): for 0 <= n < 2^22 the float quotient n*(1/d) is within a half
// of n/d, so its truncation is off by at most one, which one compare fixes.
struct DivR {
  int d;
  float r;
};
__device__ __forceinline__ DivR div_by(int d) { return DivR{d, 1.0f / (float)d}; }
__device__ __forceinline__ int quot(int n, DivR D) {
  int q = (int)((float)n * D.r);
  const int rem = n - q * D.d;
  if (rem >= D.d) ++q;
  else if (rem < 0) --q;
  return q;
}

// ------------------------------------------------------------------------
// Shared-memory addressing of one x row in the XY kernels (padded so the
// digit-reversed column reads of the r2c step are bank-conflict free).
__device__ __forceinline__ int xpos(const VolPlan& P, int e) {
  return e + (e >> P.padShift);
}

// ------------------------------------------------------------------------
// One register pass (radix R) over a set of lines in shared memory.
//   DIR = -1: decimation-in-frequency forward pass (DFT, then twiddle).
//   DIR = +1: decimation-in-time inverse pass (conjugate twiddle, then DFT).
// Lines are enumerated by l in [0, nlines); line l starts at
// lbase(l) = (l / l0n) * s1 + (l % l0n) * s0; element e of a line sits at
// lbase + e * es, mapped through xpos() when PADX is true.
// Work items: (line, block b < n/len, i < span).  If l0fast, consecutive
// threads take consecutive l0 (lines adjacent in memory); otherwise
// consecutive i.
template <int R, int DIR, bool PADX>
__device__ __forceinline__ void smem_pass(float2* sm, const VolPlan& P,
                                          const AxisPlan& A, int s, int nlines,
                                          int l0n, int s0, int s1, int es,
                                          bool l0fast, const float2* CLARITY_RESTRICT tw) {
  const int n = A.n;
  const int len = A.len[s];
  const int span = A.span[s];
  const int nblk = n / len;
  const int per_line = nblk * span;  // = n / R
  const int total = nlines * per_line;
  const int twstep = n / len;
  const DivR Dl0 = div_by(l0n), Dpl = div_by(per_line), Dsp = div_by(span);
  for (int f = threadIdx.x; f < total; f += blockDim.x) {
    int l, rem, lq, lr;  // line l = lq*l0n + lr
    if (l0fast) {
      const int rest = quot(f, Dl0);
      lr = f - rest * l0n;
      lq = quot(rest, Dpl);
      rem = rest - lq * per_line;
      l = lq * l0n + lr;
    } else {
      l = quot(f, Dpl);
      rem = f - l * per_line;
      lq = quot(l, Dl0);
      lr = l - lq * l0n;
    }
    const int b = quot(rem, Dsp);
    const int i = rem - b * span;
    const int lb = lq * s1 + lr * s0;
    const int e0 = b * len + i;
    float2 v[R];
#pragma unroll
    for (int t = 0; t < R; ++t) {
      const int e = e0 + t * span;
      v[t] = sm[lb + (PADX ? xpos(P, e) : e) * es];
    }
    if constexpr (DIR < 0) {
      dft<R, -1>(v);
      if (i != 0) {
#pragma unroll
        for (int k = 1; k < R; ++k) v[k] = cmul(v[k], CLARITY_LDG(&tw[i * k * twstep]));
      }
    } else {
      if (i != 0) {
#pragma unroll
        for (int k = 1; k < R; ++k) v[k] = cmulc(v[k], CLARITY_LDG(&tw[i * k * twstep]));
      }
      dft<R, +1>(v);
    }
#pragma unroll
    for (int t = 0; t < R; ++t) {
      const int e = e0 + t * span;
      sm[lb + (PADX ? xpos(P, e) : e) * es] = v[t];
    }
  }
}

template <int DIR, bool PADX>
__device__ __noinline__ void smem_pass_rt(float2* sm, const VolPlan& P,
                                          const AxisPlan& A, int s, int nlines,
                                          int l0n, int s0, int s1, int es,
                                          bool l0fast, const float2* tw) {
  switch (A.radix[s]) {
#define CLARITY_PASS_CASE(RR)                                              \
  case RR:                                                                 \
    smem_pass<RR, DIR, PADX>(sm, P, A, s, nlines, l0n, s0, s1, es, l0fast, \
                             tw);                                          \
    break;
    CLARITY_FOR_EACH_RADIX(CLARITY_PASS_CASE)
#undef CLARITY_PASS_CASE
    default:
      break;
  }
}

// Forward (DIF) passes first..npass-1 of axis A over lines in smem.
template <bool PADX>
__device__ __forceinline__ void smem_forward(float2* sm, const VolPlan& P,
                                             const AxisPlan& A, int first,
                                             int nlines, int l0n, int s0,
                                             int s1, int es, bool l0fast,
                                             const float2* tw) {
  for (int s = first; s < A.npass; ++s) {
    smem_pass_rt<-1, PADX>(sm, P, A, s, nlines, l0n, s0, s1, es, l0fast, tw);
    __syncthreads();
  }
}

// Inverse (DIT) passes npass-1 down to last of axis A.
template <bool PADX>
__device__ __forceinline__ void smem_inverse(float2* sm, const VolPlan& P,
                                             const AxisPlan& A, int last,
                                             int nlines, int l0n, int s0,
                                             int s1, int es, bool l0fast,
                                             const float2* tw) {
  for (int s = A.npass - 1; s >= last; --s) {
    smem_pass_rt<+1, PADX>(sm, P, A, s, nlines, l0n, s0, s1, es, l0fast, tw);
    __syncthreads();
  }
}

// ------------------------------------------------------------------------
// XY pass, first x register pass: read rows straight from HBM through the
// prologue, DIF radix R, write to smem.  Row r of the tile is
// (g, j) = (r / Ay, r % Ay) -> y = y0base + g + By*j.
template <int R, class Pro>
__device__ __forceinline__ void x_first_pass(float2* sm, const VolPlan& P,
                                             const Pro& pro, int z, int y0base,
                                             const float2* CLARITY_RESTRICT tw) {
  const AxisPlan& A = P.ax;
  const int span = A.span[0];
  const int rows = P.G * P.Ay;
  const int total = rows * span;
  const DivR Dsp = div_by(span), Day = div_by(P.Ay);
  for (int f = threadIdx.x; f < total; f += blockDim.x) {
    const int r = quot(f, Dsp);
    const int i = f - r * span;
    const int g = quot(r, Day), j = r - g * P.Ay;
    const int y = y0base + g + P.By * j;
    float2 v[R];
#pragma unroll
    for (int t = 0; t < R; ++t) v[t] = pro.load_c(i + t * span, y, z);
    dft<R, -1>(v);
    if (i != 0) {
#pragma unroll
      for (int k = 1; k < R; ++k) v[k] = cmul(v[k], CLARITY_LDG(&tw[i * k]));
    }
    float2* row = sm + r * P.rowStride;
#pragma unroll
    for (int t = 0; t < R; ++t) row[xpos(P, i + t * span)] = v[t];
  }
}

// Single-element variant for a length-1 x axis (nx = 2, even mode).
template <class Pro>
__device__ __forceinline__ void x_load_only(float2* sm, const VolPlan& P,
                                            const Pro& pro, int z, int y0base) {
  const int rows = P.G * P.Ay;
  const int total = rows * P.M;
  const DivR Dm = div_by(P.M), Day = div_by(P.Ay);
  for (int f = threadIdx.x; f < total; f += blockDim.x) {
    const int r = quot(f, Dm);
    const int m = f - r * P.M;
    const int g = quot(r, Day), j = r - g * P.Ay;
    const int y = y0base + g + P.By * j;
    sm[r * P.rowStride + xpos(P, m)] = pro.load_c(m, y, z);
  }
}

// ------------------------------------------------------------------------
// The r2c column step + length-Ay DFT, writing the S layout.
// Work item it < P.items for row group g:
//   even mode: it == 0 handles kx = 0, M (and M/2 when M is even);
//              it >= 1 handles the pair (it, M - it);
//   odd mode:  item it is the single column kx = it.
// Offset of S[0][kg][z][y0][ki] (kx = kg*W + ki); k1 adds k1_stride(P).
__device__ __forceinline__ unsigned s_base(const VolPlan& P, int kx, int z, int y0) {
  const int kg = kx / P.W, ki = kx - kg * P.W;
  return (((unsigned)kg * P.nz + z) * P.By + y0) * P.W + ki;
}
__device__ __forceinline__ unsigned k1_stride(const VolPlan& P) {
  return (unsigned)P.KG * P.nz * P.By * P.W;
}

template <int AY>
__device__ __forceinline__ void col_split_store(float2* v, const VolPlan& P,
                                                float2* CLARITY_RESTRICT S, int kx,
                                                int z, int y0,
                                                const float2* CLARITY_RESTRICT twny) {
  dft<AY, -1>(v);
  float2* dst = S + s_base(P, kx, z, y0);
  const unsigned ks = k1_stride(P);
#pragma unroll
  for (int k1 = 0; k1 < AY; ++k1) {
    float2 w = (k1 == 0 || y0 == 0) ? make_float2(1.f, 0.f)
                                    : CLARITY_LDG(&twny[y0 * k1]);
    dst[k1 * ks] = cmul(v[k1], w);
  }
}

template <int AY>
__device__ __forceinline__ void r2c_cols_forward(const float2* sm,
                                                 const VolPlan& P,
                                                 float2* CLARITY_RESTRICT S, int z,
                                                 int y0base,
                                                 const float2* CLARITY_RESTRICT tw,
                                                 const int* CLARITY_RESTRICT xrev) {
  const float2* twr = tw + P.tw_r2c_off;
  const float2* twny = tw + P.tw_ny_off;
  const int total = P.G * P.items;
  const DivR Dg = div_by(P.G);
  for (int f = threadIdx.x; f < total; f += blockDim.x) {
    const int it = quot(f, Dg);
    const int g = f - it * P.G;
    const int y0 = y0base + g;
    const float2* rows = sm + (g * AY) * P.rowStride;
    if (P.xmode == 1) {
      const int pk = xpos(P, CLARITY_LDG(&xrev[it]));
      float2 a[AY];
#pragma unroll
      for (int j = 0; j < AY; ++j) a[j] = rows[j * P.rowStride + pk];
      col_split_store<AY>(a, P, S, it, z, y0, twny);
      continue;
    }
    const int M = P.M;
    if (it == 0) {
      const int p0 = xpos(P, 0);
#pragma unroll 1
      for (int side = 0; side < 2; ++side) {
        float2 xc[AY];
#pragma unroll
        for (int j = 0; j < AY; ++j) {
          const float2 Z0 = rows[j * P.rowStride + p0];
          xc[j] = make_float2(side == 0 ? Z0.x + Z0.y : Z0.x - Z0.y, 0.f);
        }
        col_split_store<AY>(xc, P, S, side == 0 ? 0 : M, z, y0, twny);
      }
      if ((M & 1) == 0 && M >= 2) {
        const int ph = xpos(P, CLARITY_LDG(&xrev[M / 2]));
        float2 xh[AY];
#pragma unroll
        for (int j = 0; j < AY; ++j) xh[j] = conjf2(rows[j * P.rowStride + ph]);
        col_split_store<AY>(xh, P, S, M / 2, z, y0, twny);
      }
    } else {
      // pair (k, M-k); one output column at a time keeps register use at
      // one column of Ay values
      const int k = it;
      const int pa = xpos(P, CLARITY_LDG(&xrev[k]));
      const int pb = xpos(P, CLARITY_LDG(&xrev[M - k]));
      const float2 w = CLARITY_LDG(&twr[k]);
#pragma unroll 1
      for (int side = 0; side < 2; ++side) {
        float2 xc[AY];
#pragma unroll
        for (int j = 0; j < AY; ++j) {
          const float2 a = rows[j * P.rowStride + pa];
          const float2 b = conjf2(rows[j * P.rowStride + pb]);
          const float2 e = make_float2(0.5f * (a.x + b.x), 0.5f * (a.y + b.y));
          // o = (a - b) / (2i) = (a - b) * (-i/2)
          const float2 d = csub(a, b);
          const float2 o = make_float2(0.5f * d.y, -0.5f * d.x);
          const float2 wo = cmul(w, o);
          xc[j] = side == 0 ? cadd(e, wo) : conjf2(csub(e, wo));
        }
        col_split_store<AY>(xc, P, S, side == 0 ? k : M - k, z, y0, twny);
      }
    }
  }
}

// Inverse: read the S layout, inverse split twiddle, inverse length-Ay DFT,
// c2r pre-processing, write digit-reversed rows into smem.
template <int AY>
__device__ __forceinline__ void col_split_load(float2* v, const VolPlan& P,
                                               const float2* CLARITY_RESTRICT S,
                                               int kx, int z, int y0,
                                               const float2* CLARITY_RESTRICT twny) {
  const float2* src = S + s_base(P, kx, z, y0);
  const unsigned ks = k1_stride(P);
#pragma unroll
  for (int k1 = 0; k1 < AY; ++k1) {
    float2 a = CLARITY_LDG(&src[k1 * ks]);
    if (k1 != 0 && y0 != 0) a = cmulc(a, CLARITY_LDG(&twny[y0 * k1]));
    v[k1] = a;
  }
  dft<AY, +1>(v);
}

template <int AY>
__device__ __forceinline__ void c2r_cols_inverse(float2* sm, const VolPlan& P,
                                                 const float2* CLARITY_RESTRICT S,
                                                 int z, int y0base,
                                                 const float2* CLARITY_RESTRICT tw,
                                                 const int* CLARITY_RESTRICT xrev) {
  const float2* twr = tw + P.tw_r2c_off;
  const float2* twny = tw + P.tw_ny_off;
  const int total = P.G * P.items;
  const DivR Dg = div_by(P.G);
  for (int f = threadIdx.x; f < total; f += blockDim.x) {
    const int it = quot(f, Dg);
    const int g = f - it * P.G;
    const int y0 = y0base + g;
    float2* rows = sm + (g * AY) * P.rowStride;
    if (P.xmode == 1) {
      const int pk = xpos(P, CLARITY_LDG(&xrev[it]));
      float2 a[AY];
      col_split_load<AY>(a, P, S, it, z, y0, twny);
#pragma unroll
      for (int j = 0; j < AY; ++j) rows[j * P.rowStride + pk] = a[j];
      continue;
    }
    const int M = P.M;
    if (it == 0) {
      const int p0 = xpos(P, 0);
      {
        float2 xc[AY];
        col_split_load<AY>(xc, P, S, 0, z, y0, twny);
#pragma unroll
        for (int j = 0; j < AY; ++j) rows[j * P.rowStride + p0] = xc[j];
      }
      {
        float2 xm[AY];
        col_split_load<AY>(xm, P, S, M, z, y0, twny);
#pragma unroll
        for (int j = 0; j < AY; ++j) {
          // imaginary parts of the self-conjugate bins are ignored (FFTW c2r)
          const float x0 = rows[j * P.rowStride + p0].x;
          rows[j * P.rowStride + p0] = make_float2(x0 + xm[j].x, x0 - xm[j].x);
        }
      }
      if ((M & 1) == 0 && M >= 2) {
        float2 xh[AY];
        col_split_load<AY>(xh, P, S, M / 2, z, y0, twny);
        const int ph = xpos(P, CLARITY_LDG(&xrev[M / 2]));
#pragma unroll
        for (int j = 0; j < AY; ++j)
          rows[j * P.rowStride + ph] = make_float2(2.f * xh[j].x, -2.f * xh[j].y);
      }
    } else {
      // pair (k, M-k): inverse-transform each column into its own smem
      // slot, then combine the two slots in place (same thread, no sync)
      const int k = it;
      const int pa = xpos(P, CLARITY_LDG(&xrev[k]));
      const int pb = xpos(P, CLARITY_LDG(&xrev[M - k]));
      {
        float2 xc[AY];
        col_split_load<AY>(xc, P, S, k, z, y0, twny);
#pragma unroll
        for (int j = 0; j < AY; ++j) rows[j * P.rowStride + pa] = xc[j];
      }
      {
        float2 xc[AY];
        col_split_load<AY>(xc, P, S, M - k, z, y0, twny);
#pragma unroll
        for (int j = 0; j < AY; ++j) rows[j * P.rowStride + pb] = xc[j];
      }
      const float2 w = CLARITY_LDG(&twr[k]);
#pragma unroll 4
      for (int j = 0; j < AY; ++j) {
        const float2 xa = rows[j * P.rowStride + pa];
        const float2 b = conjf2(rows[j * P.rowStride + pb]);
        const float2 e = cadd(xa, b);
        const float2 o = cmulc(csub(xa, b), w);  // (a - b) * conj(w)
        // Z[k] = e + i o ; Z[M-k] = conj(e) + i conj(o)
        rows[j * P.rowStride + pa] = make_float2(e.x - o.y, e.y + o.x);
        rows[j * P.rowStride + pb] = make_float2(e.x + o.y, -e.y + o.x);
      }
    }
  }
}

template <bool FWD>
__device__ __noinline__ void cols_rt(float2* sm, const VolPlan& P, float2* S,
                                     int z, int y0base, const float2* tw,
                                     const int* xrev) {
  switch (P.Ay) {
#define CLARITY_COL_CASE(RR)                                           \
  case RR:                                                             \
    if constexpr (FWD)                                                 \
      r2c_cols_forward<RR>(sm, P, S, z, y0base, tw, xrev);            \
    else                                                               \
      c2r_cols_inverse<RR>(sm, P, S, z, y0base, tw, xrev);            \
    break;
    CLARITY_COL_CASE(1)
    CLARITY_FOR_EACH_RADIX(CLARITY_COL_CASE)
#undef CLARITY_COL_CASE
    default:
      break;
  }
}

// ------------------------------------------------------------------------
// Last inverse x pass (DIT pass 0) straight into the epilogue: the thread
// holds complex row elements m = i + span*t, i.e. reals x = 2m, 2m+1 (even
// mode) or x = m (odd mode).  Epi::store(x_even, y, z, v) receives the
// complex value; FUSE re-applies the forward DIF pass 0 to what the
// epilogue returns and writes it back to smem.
template <int R, class Epi, bool FUSE>
__device__ __forceinline__ void x_last_pass(float2* sm, const VolPlan& P,
                                            Epi& epi, int z, int y0base,
                                            const float2* CLARITY_RESTRICT tw) {
  const AxisPlan& A = P.ax;
  const int span = A.npass > 0 ? A.span[0] : 1;
  const int rows = P.G * P.Ay;
  const int total = rows * span;
  const DivR Dsp = div_by(span), Day = div_by(P.Ay);
  for (int f = threadIdx.x; f < total; f += blockDim.x) {
    const int r = quot(f, Dsp);
    const int i = f - r * span;
    const int g = quot(r, Day), j = r - g * P.Ay;
    const int y = y0base + g + P.By * j;
    float2* row = sm + r * P.rowStride;
    float2 v[R];
#pragma unroll
    for (int t = 0; t < R; ++t) v[t] = row[xpos(P, i + t * span)];
    if (A.npass > 0) {
      if (i != 0) {
#pragma unroll
        for (int k = 1; k < R; ++k) v[k] = cmulc(v[k], CLARITY_LDG(&tw[i * k]));
      }
      dft<R, +1>(v);
    }
#pragma unroll
    for (int t = 0; t < R; ++t) v[t] = epi.apply_c(i + t * span, y, z, v[t]);
    if constexpr (FUSE) {
      if (A.npass > 0) {
        dft<R, -1>(v);
        if (i != 0) {
#pragma unroll
          for (int k = 1; k < R; ++k) v[k] = cmul(v[k], CLARITY_LDG(&tw[i * k]));
        }
      }
#pragma unroll
      for (int t = 0; t < R; ++t) row[xpos(P, i + t * span)] = v[t];
    }
  }
}

template <class Epi, bool FUSE>
__device__ __forceinline__ void x_last_pass_rt(float2* sm, const VolPlan& P,
                                               Epi& epi, int z, int y0base,
                                               const float2* tw) {
  if (P.ax.npass == 0) {
    x_last_pass<1, Epi, FUSE>(sm, P, epi, z, y0base, tw);
    return;
  }
  switch (P.ax.radix[0]) {
#define CLARITY_LAST_CASE(RR)                                  \
  case RR:                                                     \
    x_last_pass<RR, Epi, FUSE>(sm, P, epi, z, y0base, tw);     \
    break;
    CLARITY_FOR_EACH_RADIX(CLARITY_LAST_CASE)
#undef CLARITY_LAST_CASE
    default:
      break;
  }
}

template <class Pro>
__device__ __forceinline__ void x_first_pass_rt(float2* sm, const VolPlan& P,
                                                const Pro& pro, int z,
                                                int y0base, const float2* tw) {
  if (P.ax.npass == 0) {
    x_load_only(sm, P, pro, z, y0base);
    return;
  }
  switch (P.ax.radix[0]) {
#define CLARITY_FIRST_CASE(RR)                              \
  case RR:                                                  \
    x_first_pass<RR, Pro>(sm, P, pro, z, y0base, tw);       \
    break;
    CLARITY_FOR_EACH_RADIX(CLARITY_FIRST_CASE)
#undef CLARITY_FIRST_CASE
    default:
      break;
  }
}

// ------------------------------------------------------------------------
// Pass bodies.  XY bodies take one (z, y0 group) tile, bid over
// z = bid / (By/G), y0base = (bid % (By/G)) * G; Z bodies take the tile
// S[k1][kg] at bid = k1*KG + kg.  The kernels below run one body per block
// (bid = blockIdx.x); the persistent batched kernel (kern_batch.cu) runs
// many, one per work item.
template <class Pro>
__device__ __forceinline__ void xy_forward_body(float2* sm, const VolPlan& P, const Pro& pro,
                                                float2* CLARITY_RESTRICT S,
                                                const float2* CLARITY_RESTRICT tw,
                                                const int* CLARITY_RESTRICT xrev, int bid) {
  const int ngroups = P.By / P.G;
  const int z = bid / ngroups;
  const int y0base = (bid - z * ngroups) * P.G;
  const float2* twx = tw + P.ax.tw_off;
  x_first_pass_rt(sm, P, pro, z, y0base, twx);
  __syncthreads();
  smem_forward<true>(sm, P, P.ax, 1, P.G * P.Ay, P.G * P.Ay, P.rowStride, 0, 1, false, twx);
  cols_rt<true>(sm, P, S, z, y0base, tw, xrev);
  pro.finish();
}

template <class Epi>
__device__ __forceinline__ void xy_inverse_body(float2* sm, const VolPlan& P, Epi& epi,
                                                const float2* CLARITY_RESTRICT S,
                                                const float2* CLARITY_RESTRICT tw,
                                                const int* CLARITY_RESTRICT xrev, int bid) {
  const int ngroups = P.By / P.G;
  const int z = bid / ngroups;
  const int y0base = (bid - z * ngroups) * P.G;
  const float2* twx = tw + P.ax.tw_off;
  cols_rt<false>(sm, P, const_cast<float2*>(S), z, y0base, tw, xrev);
  __syncthreads();
  smem_inverse<true>(sm, P, P.ax, 1, P.G * P.Ay, P.G * P.Ay, P.rowStride, 0, 1, false, twx);
  x_last_pass_rt<Epi, false>(sm, P, epi, z, y0base, twx);
  epi.finish();
}

// Inverse x/y transform, point-wise operation, forward transform: one pass.
// Reads and writes S in place (each tile owns its (z, y0-group) slice).
template <class Mid>
__device__ __forceinline__ void xy_inv_fwd_body(float2* sm, const VolPlan& P, Mid& mid,
                                                float2* CLARITY_RESTRICT S,
                                                const float2* CLARITY_RESTRICT tw,
                                                const int* CLARITY_RESTRICT xrev, int bid) {
  const int ngroups = P.By / P.G;
  const int z = bid / ngroups;
  const int y0base = (bid - z * ngroups) * P.G;
  const float2* twx = tw + P.ax.tw_off;
  // a plane whose result is known to be zero is neither read nor written;
  // the next Z pass reads those planes as zeros (Mod::zn)
  if (mid.zero_plane(z)) {
    if constexpr (requires { mid.finish_skipped(); }) mid.finish_skipped();
    return;
  }
  cols_rt<false>(sm, P, S, z, y0base, tw, xrev);
  __syncthreads();
  smem_inverse<true>(sm, P, P.ax, 1, P.G * P.Ay, P.G * P.Ay, P.rowStride, 0, 1, false, twx);
  x_last_pass_rt<Mid, true>(sm, P, mid, z, y0base, twx);
  __syncthreads();
  smem_forward<true>(sm, P, P.ax, 1, P.G * P.Ay, P.G * P.Ay, P.rowStride, 0, 1, false, twx);
  cols_rt<true>(sm, P, S, z, y0base, tw, xrev);
  mid.finish();
}

// Z pass.  Tile = S[k1][kg] (nz*By*W contiguous float2), laid out in smem as
// [z][y0][ki].  Mod::forward_only selects "transform and store" (used for the
// OTF and the Wiener numerator); otherwise Mod::apply(idx, v) runs between the
// forward and inverse transforms, idx being the element's offset in S.
template <class Mod>
__device__ __forceinline__ void z_body(float2* sm, const VolPlan& P, const Mod& mod,
                                       const float2* CLARITY_RESTRICT Sin,
                                       float2* CLARITY_RESTRICT Sout,
                                       const float2* CLARITY_RESTRICT tw, int bid) {
  const long long tile = (long long)P.nz * P.By * P.W;
  const long long base = (long long)bid * tile;
  // load (16-byte vectors when the tile size is even, which keeps every
  // tile base 16-byte aligned)
  // planes z >= zn of the input are zero (not read)
  const long long live = (long long)(mod.zn < P.nz ? mod.zn : P.nz) * P.By * P.W;
  if ((tile & 1) == 0 && (live & 1) == 0) {
    const float4* src = reinterpret_cast<const float4*>(Sin + base);
    float4* dst = reinterpret_cast<float4*>(sm);
    const int n4 = (int)(tile / 2), live4 = (int)(live / 2);
    for (int t = threadIdx.x; t < n4; t += blockDim.x)
      dst[t] = t < live4 ? CLARITY_LDG(&src[t]) : make_float4(0.f, 0.f, 0.f, 0.f);
  } else {
    for (int t = threadIdx.x; t < tile; t += blockDim.x)
      sm[t] = t < live ? Sin[base + t] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  const int BW = P.By * P.W;
  const float2* twy = tw + P.ayB.tw_off;
  const float2* twz = tw + P.az.tw_off;
  // y0 DFT: lines (z, ki), elements y0 with stride W
  smem_forward<false>(sm, P, P.ayB, 0, P.nz * P.W, P.W, 1, BW, P.W, true, twy);
  // z DFT: lines (y0, ki) = BW contiguous lines, elements z with stride BW
  smem_forward<false>(sm, P, P.az, 0, BW, BW, 1, 0, BW, true, twz);
  if (!Mod::forward_only) {
    for (int t = threadIdx.x; t < tile; t += blockDim.x)
      sm[t] = mod.apply(base + t, sm[t]);
    __syncthreads();
    smem_inverse<false>(sm, P, P.az, 0, BW, BW, 1, 0, BW, true, twz);
    smem_inverse<false>(sm, P, P.ayB, 0, P.nz * P.W, P.W, 1, BW, P.W, true, twy);
  }
  // planes z >= zout are not needed downstream: not stored
  const long long out = (long long)(mod.zout < P.nz ? mod.zout : P.nz) * P.By * P.W;
  if ((tile & 1) == 0 && (out & 1) == 0) {
    float4* dst = reinterpret_cast<float4*>(Sout + base);
    const float4* src = reinterpret_cast<const float4*>(sm);
    const int n4 = (int)(out / 2);
    for (int t = threadIdx.x; t < n4; t += blockDim.x) dst[t] = src[t];
  } else {
    for (int t = threadIdx.x; t < out; t += blockDim.x) Sout[base + t] = sm[t];
  }
}

// ------------------------------------------------------------------------
// Kernels: one body per block.  Each instance is compiled in exactly one
// translation unit (the kern_*.cu file of its family, which defines it
// explicitly); other units name it through CLARITY_EXTERN_PASS_KERNELS.  Two
// compiled copies of one kernel (say one with scalar and one with paired
// FP32 adds) would both register for the same launch and the runtime would
// run either, so results could differ between processes.
// Blocks per SM the runtime-planned kernels' register budget is sized for.
#ifndef CLARITY_GEN_MINB
#define CLARITY_GEN_MINB 2
#endif

template <class Pro>
__global__ void __launch_bounds__(256, CLARITY_GEN_MINB)
    k_xy_forward(const VolPlan P, const Pro pro, float2* CLARITY_RESTRICT S,
                 const float2* CLARITY_RESTRICT tw, const int* CLARITY_RESTRICT xrev) {
  CLARITY_DYN_SMEM(float2, sm);
  xy_forward_body(sm, P, pro, S, tw, xrev, (int)blockIdx.x);
}

template <class Epi>
__global__ void __launch_bounds__(256, CLARITY_GEN_MINB)
    k_xy_inverse(const VolPlan P, Epi epi, const float2* CLARITY_RESTRICT S,
                 const float2* CLARITY_RESTRICT tw, const int* CLARITY_RESTRICT xrev) {
  CLARITY_DYN_SMEM(float2, sm);
  xy_inverse_body(sm, P, epi, S, tw, xrev, (int)blockIdx.x);
}

template <class Mid>
__global__ void __launch_bounds__(256, CLARITY_GEN_MINB)
    k_xy_inv_fwd(const VolPlan P, Mid mid, float2* CLARITY_RESTRICT S,
                 const float2* CLARITY_RESTRICT tw, const int* CLARITY_RESTRICT xrev) {
  CLARITY_DYN_SMEM(float2, sm);
  xy_inv_fwd_body(sm, P, mid, S, tw, xrev, (int)blockIdx.x);
}

template <class Mod>
__global__ void __launch_bounds__(256, CLARITY_GEN_MINB)
    k_z(const VolPlan P, const Mod mod, const float2* CLARITY_RESTRICT Sin,
        float2* CLARITY_RESTRICT Sout, const float2* CLARITY_RESTRICT tw) {
  CLARITY_DYN_SMEM(float2, sm);
  z_body(sm, P, mod, Sin, Sout, tw, (int)blockIdx.x);
}

// The generic pass kernels the no-allocation convolution (noalloc.cu)
// launches, defined in kern_xy_fwd.cu, kern_z.cu and kern_xy_inv.cu.
#define CLARITY_EXTERN_PASS_KERNELS                                                           \
  extern template __global__ void k_xy_forward<ProPadded>(const VolPlan, const ProPadded,     \
                                                          float2*, const float2*, const int*); \
  extern template __global__ void k_xy_forward<ProImage>(const VolPlan, const ProImage,       \
                                                         float2*, const float2*, const int*);  \
  extern template __global__ void k_z<ModForward>(const VolPlan, const ModForward,            \
                                                  const float2*, float2*, const float2*);      \
  extern template __global__ void k_z<ModOTF>(const VolPlan, const ModOTF, const float2*,     \
                                              float2*, const float2*);                         \
  extern template __global__ void k_xy_inverse<EpiClip>(const VolPlan, EpiClip, const float2*, \
                                                        const float2*, const int*);

}  // namespace clarity
