// passes_static.cuh -- the fused FFT pass kernels specialised at compile time
// for the work-box shapes that matter most (the benchmark and test
// configurations).  Same data layout, digit orders and twiddle tables as the
// runtime-generic kernels in passes.cuh (the planner produces identical
// plans), so the two paths can be mixed freely; here every radix, stride and
// divisor is a constant, the x digit-reversal is computed instead of looked
// up, and the spectral operation of the Z pass is fused into its last
// forward / first inverse register pass.
#pragma once
#include "dft_codelets.cuh"
#include "launch_macro.cuh"
#include "plan.hpp"
#include "tc_dft.cuh"
#include "tma.cuh"

// Blocks per SM the XY kernels' register budget is sized for (a build
// option; 3 trades a few spills for occupancy and measured faster than 2).
#ifndef CLARITY_XY_MINBLOCKS
#define CLARITY_XY_MINBLOCKS 3
#endif

namespace clarity {
namespace st {

// DIF radix sequence of one axis (1 = pass unused).
template <int R0, int R1 = 1, int R2 = 1>
struct Rad {
  static constexpr int n = R0 * R1 * R2;
  static constexpr int npass = (R0 > 1) + (R1 > 1) + (R2 > 1);
  static constexpr int radix(int s) { return s == 0 ? R0 : (s == 1 ? R1 : R2); }
  static constexpr int len(int s) { return s == 0 ? n : (s == 1 ? n / R0 : n / (R0 * R1)); }
  static constexpr int span(int s) { return len(s) / radix(s); }
};

constexpr int ctz_c(int v) {
  int c = 0;
  while (v > 1 && !(v & 1)) { v >>= 1; ++c; }
  return c;
}

// Even nx only (half-length complex rows).  T_ threads per block: 256 where
// several blocks fit an SM; the boxes whose XY and z tiles take most of an
// SM's shared memory (one block per SM) use more threads, so the SM still
// holds enough warps to hide shared-memory and HBM latency.  TZ_: the same
// for the FP32 z kernel (launched as ZThreads<SH>, the shape with TZ_ threads).
template <class XR, int AY_, class YR, class ZR, int G_, int W_, int T_ = 256, int TZ_ = T_>
struct Shape {
  using X = XR;
  using Y = YR;
  using Z = ZR;
  static constexpr int M = X::n, AY = AY_, BY = Y::n, NZ = Z::n, G = G_, W = W_;
  static constexpr int NX = 2 * M, NY = AY * BY;
  static constexpr int XS = M + 1, KG = (XS + W - 1) / W;
  static constexpr int PADSHIFT =
      (X::npass <= 1 || (X::span(0) & 1)) ? 30 : ctz_c(X::span(0));
  static constexpr int ROWSTRIDE_RAW = (M - 1) + ((M - 1) >> PADSHIFT) + 1;
  static constexpr int ROWSTRIDE = (ROWSTRIDE_RAW % 2 == 0) ? ROWSTRIDE_RAW + 1 : ROWSTRIDE_RAW;
  static constexpr int ROWS = G * AY;
  // Row groups g are GSTRIDE apart: AY*ROWSTRIDE plus 8 float2 when that is
  // a multiple of 16, so the column step's groups use disjoint banks.
  static constexpr int GSTRIDE = AY * ROWSTRIDE + (((AY * ROWSTRIDE) % 16 == 0) ? 8 : 0);
  static constexpr int ITEMS = (M % 2 == 0) ? (M / 2 > 1 ? M / 2 : 1) : (M + 1) / 2;
  static constexpr int BW = BY * W;
  static constexpr int TILE = NZ * BW;
  static constexpr int THREADS = T_;
  static constexpr int Z_THREADS = TZ_;
  static_assert(T_ % 32 == 0 && T_ >= 256 && T_ <= 1024, "whole warps, 256..1024 threads");
  // blocks per SM the register budget is sized for (__launch_bounds__)
  static constexpr int XY_MINB = T_ == 256 ? CLARITY_XY_MINBLOCKS : 1;
  static constexpr int Z_MINB = T_ == 256 ? 2 : 1;
  static constexpr int XY_SMEM = G * GSTRIDE * 8;
  static constexpr int Z_SMEM = TILE * 8;
  static constexpr int NGROUPS = BY / G;
  // Z kernel with one register pass per y0 line (BY <= 32): padded z stride
  // ZS = BW + W keeps both the per-line y0 accesses and the z passes free of
  // bank conflicts.
  static constexpr bool Y_PER_LINE = BY <= 32;
  static constexpr int ZS = BW + W;
  // padded tile, then the z twiddle table w_nz^t (NZ entries)
  static constexpr int Z2_TILE_BYTES = NZ * ZS * 8;
  static constexpr int Z2_SMEM = Z2_TILE_BYTES + NZ * 8;
};

// Shape SH with TZ_ threads for every kernel: the FP32 z kernel's launch shape.
template <class SH>
using ZThreads = Shape<typename SH::X, SH::AY, typename SH::Y, typename SH::Z, SH::G, SH::W,
                       SH::Z_THREADS, SH::Z_THREADS>;

template <class SH>
__device__ __forceinline__ int xp(int e) {
  return e + (e >> SH::PADSHIFT);
}

// Shared-memory offset of tile row r = g*AY + j.
template <class SH>
__device__ __forceinline__ int row_off(int r) {
  const int g = r / SH::AY, j = r - g * SH::AY;
  return g * SH::GSTRIDE + j * SH::ROWSTRIDE;
}

// Digit-reversed slot of natural x frequency k after the DIF passes.
template <class SH>
__device__ __forceinline__ int xrev(int k) {
  using X = typename SH::X;
  int pos = 0, rem = k;
#pragma unroll
  for (int s = 0; s < X::npass; ++s) {
    const int d = rem % X::radix(s);
    rem /= X::radix(s);
    pos += d * X::span(s);
  }
  return pos;
}

// Offset of S[0][kg][z][y0][ki] for kx = kg*W + ki; k1 adds K1STRIDE.
template <class SH>
__device__ __forceinline__ unsigned sbase(int kx, int z, int y0) {
  const int kg = kx / SH::W, ki = kx % SH::W;
  return (((unsigned)kg * SH::NZ + z) * SH::BY + y0) * SH::W + ki;
}
template <class SH>
constexpr unsigned kK1Stride = (unsigned)SH::KG * SH::NZ * SH::BY * SH::W;

// ------------------------------------------------------------------ x rows
// One register pass S of the x axis over all rows of the XY tile.
// Row predicates: rows whose content is known to be zero are not transformed.
struct NoSkip {
  __device__ __forceinline__ bool operator()(int) const { return false; }
};
template <class SH, class F>
struct RowSkip {
  const F& f;
  int z, y0base;
  __device__ __forceinline__ bool operator()(int r) const {
    const int g = r / SH::AY, j = r - g * SH::AY;
    return f.zero_row(y0base + g + SH::BY * j, z);
  }
};

// Tile rows visited by a pass: all G*AY rows, or (COMPACT) only the first
// L rows j < L of each group, so threads are not left idle on rows whose
// content is known to be zero.
template <class SH, bool COMPACT>
__device__ __forceinline__ int visit_rows(int L) {
  return COMPACT ? SH::G * L : SH::ROWS;
}
template <class SH, bool COMPACT>
__device__ __forceinline__ int visit_row(int rv, int L) {
  if constexpr (!COMPACT) return rv;
  const int g = rv / L;
  return g * SH::AY + (rv - g * L);
}

// tw: the x twiddle table w_M^t, in global or shared memory (plain loads).
template <class SH, int S, int DIR, class Skip, bool COMPACT = false>
__device__ __forceinline__ void x_pass(float2* sm, const float2* tw,
                                       const Skip& skip, int L = SH::AY) {
  using X = typename SH::X;
  constexpr int R = X::radix(S), len = X::len(S), span = len / R;
  constexpr int per_row = X::n / R, twstep = X::n / len;
  const int total = visit_rows<SH, COMPACT>(L) * per_row;
#pragma unroll 1
  for (int f = threadIdx.x; f < total; f += CLARITY_BLOCK_STRIDE(SH::THREADS)) {
    const int rv = f / per_row;
    const int r = visit_row<SH, COMPACT>(rv, L);
    if (skip(r)) continue;
    const int rem = f - rv * per_row;
    const int b = rem / span;
    const int i = rem - b * span;
    float2* row = sm + row_off<SH>(r);
    const int e0 = b * len + i;
    float2 v[R];
#pragma unroll
    for (int t = 0; t < R; ++t) v[t] = row[xp<SH>(e0 + t * span)];
    if constexpr (DIR < 0) {
      dft<R, -1>(v);
      if (span > 1 && i != 0) {
#pragma unroll
        for (int k = 1; k < R; ++k) v[k] = cmul(v[k], tw[i * k * twstep]);
      }
    } else {
      if (span > 1 && i != 0) {
#pragma unroll
        for (int k = 1; k < R; ++k) v[k] = cmulc(v[k], tw[i * k * twstep]);
      }
      dft<R, +1>(v);
    }
#pragma unroll
    for (int t = 0; t < R; ++t) row[xp<SH>(e0 + t * span)] = v[t];
  }
}

template <class SH, int S, class Skip = NoSkip, bool COMPACT = false>
__device__ __forceinline__ void x_forward_from(float2* sm, const float2* tw,
                                               const Skip& skip = Skip{}, int L = SH::AY) {
  if constexpr (S < SH::X::npass) {
    x_pass<SH, S, -1, Skip, COMPACT>(sm, tw, skip, L);
    __syncthreads();
    x_forward_from<SH, S + 1, Skip, COMPACT>(sm, tw, skip, L);
  }
}

template <class SH, int S, class Skip = NoSkip, bool COMPACT = false>
__device__ __forceinline__ void x_inverse_down_to(float2* sm, const float2* tw,
                                                  const Skip& skip = Skip{}, int L = SH::AY) {
  // inverse passes npass-1 .. S (inclusive)
  if constexpr (S < SH::X::npass) {
    x_inverse_down_to<SH, S + 1, Skip, COMPACT>(sm, tw, skip, L);
    x_pass<SH, S, +1, Skip, COMPACT>(sm, tw, skip, L);
    __syncthreads();
  }
}

// First x pass straight from HBM through the prologue.
template <class SH, class Pro>
__device__ __forceinline__ void x_first(float2* sm, const Pro& pro, int z, int y0base,
                                        const float2* __restrict__ tw) {
  using X = typename SH::X;
  constexpr int R = X::radix(0), span = X::span(0), total = SH::ROWS * span;
#pragma unroll 1
  for (int f = threadIdx.x; f < total; f += CLARITY_BLOCK_STRIDE(SH::THREADS)) {
    const int r = f / span;
    const int i = f - r * span;
    const int g = r / SH::AY, j = r - g * SH::AY;
    const int y = y0base + g + SH::BY * j;
    float2 v[R];
#pragma unroll
    for (int t = 0; t < R; ++t) v[t] = pro.load_c(i + t * span, y, z);
    dft<R, -1>(v);
    if (i != 0) {
#pragma unroll
      for (int k = 1; k < R; ++k) v[k] = cmul(v[k], __ldg(&tw[i * k]));
    }
    float2* row = sm + row_off<SH>(r);
#pragma unroll
    for (int t = 0; t < R; ++t) row[xp<SH>(i + t * span)] = v[t];
  }
}

// Last inverse x pass (pass 0) into the epilogue; FUSE re-applies forward
// pass 0 to what the epilogue returns.
template <class SH, class Epi, bool FUSE, class Skip = NoSkip, bool COMPACT = false>
__device__ __forceinline__ void x_last(float2* sm, Epi& epi, int z, int y0base,
                                       const float2* __restrict__ tw,
                                       const Skip& skip = Skip{}, int L = SH::AY) {
  using X = typename SH::X;
  constexpr int R = X::radix(0), span = X::span(0);
  const int total = visit_rows<SH, COMPACT>(L) * span;
#pragma unroll 1
  for (int f = threadIdx.x; f < total; f += CLARITY_BLOCK_STRIDE(SH::THREADS)) {
    const int rv = f / span;
    const int r = visit_row<SH, COMPACT>(rv, L);
    const int i = f - rv * span;
    const int g = r / SH::AY, j = r - g * SH::AY;
    const int y = y0base + g + SH::BY * j;
    float2* row = sm + row_off<SH>(r);
    if (skip(r)) {  // known-zero row: its forward transform is zero
      if constexpr (FUSE) {
#pragma unroll
        for (int t = 0; t < R; ++t) row[xp<SH>(i + t * span)] = make_float2(0.f, 0.f);
      }
      continue;
    }
    float2 v[R];
#pragma unroll
    for (int t = 0; t < R; ++t) v[t] = row[xp<SH>(i + t * span)];
    if (i != 0) {
#pragma unroll
      for (int k = 1; k < R; ++k) v[k] = cmulc(v[k], __ldg(&tw[i * k]));
    }
    dft<R, +1>(v);
#pragma unroll
    for (int t = 0; t < R; ++t) v[t] = epi.apply_c(i + t * span, y, z, v[t]);
    if constexpr (FUSE) {
      dft<R, -1>(v);
      if (i != 0) {
#pragma unroll
        for (int k = 1; k < R; ++k) v[k] = cmul(v[k], __ldg(&tw[i * k]));
      }
#pragma unroll
      for (int t = 0; t < R; ++t) row[xp<SH>(i + t * span)] = v[t];
    }
  }
}

// ------------------------------------------------------- r2c / c2r columns
// Column kx of the group's rows after the Ay-DFT: twiddled by w_ny^(y0*k1)
// and stored to S[k1][kx][z][y0] (store_col), or loaded and untwiddled
// (load_col) before the inverse Ay-DFT.
template <class SH>
__device__ __forceinline__ void store_col(const float2* v, float2* __restrict__ S, int kx,
                                          int z, int y0, const float2* __restrict__ twny) {
  float2* dst = S + sbase<SH>(kx, z, y0);
#pragma unroll
  for (int k1 = 0; k1 < SH::AY; ++k1) {
    const float2 w = (k1 == 0 || y0 == 0) ? make_float2(1.f, 0.f) : __ldg(&twny[y0 * k1]);
    dst[k1 * kK1Stride<SH>] = cmul(v[k1], w);
  }
}

template <class SH>
__device__ __forceinline__ void load_col(float2* v, const float2* __restrict__ S, int kx,
                                         int z, int y0, const float2* __restrict__ twny) {
  const float2* src = S + sbase<SH>(kx, z, y0);
#pragma unroll
  for (int k1 = 0; k1 < SH::AY; ++k1) {
    float2 a = __ldg(&src[k1 * kK1Stride<SH>]);
    if (k1 != 0 && y0 != 0) a = cmulc(a, __ldg(&twny[y0 * k1]));
    v[k1] = a;
  }
}

template <class SH>
__device__ __forceinline__ void split_store(float2* v, float2* __restrict__ S, int kx,
                                            int z, int y0, const float2* __restrict__ twny) {
  dft<SH::AY, -1>(v);
  store_col<SH>(v, S, kx, z, y0, twny);
}

template <class SH>
__device__ __forceinline__ void split_load(float2* v, const float2* __restrict__ S, int kx,
                                           int z, int y0, const float2* __restrict__ twny) {
  load_col<SH>(v, S, kx, z, y0, twny);
  dft<SH::AY, +1>(v);
}

template <class SH>
__device__ __forceinline__ void cols_forward(const float2* sm, float2* __restrict__ S, int z,
                                             int y0base, const float2* __restrict__ twr,
                                             const float2* __restrict__ twny) {
  constexpr int M = SH::M, AY = SH::AY, RS = SH::ROWSTRIDE;
  constexpr int total = SH::G * SH::ITEMS;
#pragma unroll 1
  for (int f = threadIdx.x; f < total; f += CLARITY_BLOCK_STRIDE(SH::THREADS)) {
    const int g = f % SH::G;
    const int it = f / SH::G;
    const int y0 = y0base + g;
    const float2* rows = sm + g * SH::GSTRIDE;
    if (it == 0) {
      // kx = 0 and kx = M have real columns a, b: one DFT of a + i b gives
      // both, A[k] = (P[k] + conj P[-k]) / 2, B[k] = (P[k] - conj P[-k]) / 2i
      const int p0 = xp<SH>(0);
      {
        float2 pk[AY];
#pragma unroll
        for (int j = 0; j < AY; ++j) {
          const float2 Z0 = rows[j * RS + p0];
          pk[j] = make_float2(Z0.x + Z0.y, Z0.x - Z0.y);
        }
        dft<AY, -1>(pk);
        float2 a[AY], b[AY];
#pragma unroll
        for (int k = 0; k < AY; ++k) {
          const float2 p = pk[k], q = pk[(AY - k) % AY];
          a[k] = make_float2(0.5f * (p.x + q.x), 0.5f * (p.y - q.y));
          b[k] = make_float2(0.5f * (p.y + q.y), 0.5f * (q.x - p.x));
        }
        store_col<SH>(a, S, 0, z, y0, twny);
        store_col<SH>(b, S, M, z, y0, twny);
      }
      if constexpr (M % 2 == 0 && M >= 2) {
        const int ph = xp<SH>(xrev<SH>(M / 2));
        float2 xh[AY];
#pragma unroll
        for (int j = 0; j < AY; ++j) xh[j] = conjf2(rows[j * RS + ph]);
        split_store<SH>(xh, S, M / 2, z, y0, twny);
      }
    } else {
      const int k = it;
      const int pa = xp<SH>(xrev<SH>(k));
      const int pb = xp<SH>(xrev<SH>(M - k));
      const float2 w = __ldg(&twr[k]);
#pragma unroll 1
      for (int side = 0; side < 2; ++side) {
        float2 xc[AY];
#pragma unroll
        for (int j = 0; j < AY; ++j) {
          const float2 a = rows[j * RS + pa];
          const float2 b = conjf2(rows[j * RS + pb]);
          const float2 e = make_float2(0.5f * (a.x + b.x), 0.5f * (a.y + b.y));
          const float2 d = csub(a, b);
          const float2 o = make_float2(0.5f * d.y, -0.5f * d.x);
          const float2 wo = cmul(w, o);
          xc[j] = side == 0 ? cadd(e, wo) : conjf2(csub(e, wo));
        }
        split_store<SH>(xc, S, side == 0 ? k : M - k, z, y0, twny);
      }
    }
  }
}

template <class SH>
__device__ __forceinline__ void cols_inverse(float2* sm, const float2* __restrict__ S, int z,
                                             int y0base, const float2* __restrict__ twr,
                                             const float2* __restrict__ twny) {
  constexpr int M = SH::M, AY = SH::AY, RS = SH::ROWSTRIDE;
  constexpr int total = SH::G * SH::ITEMS;
#pragma unroll 1
  for (int f = threadIdx.x; f < total; f += CLARITY_BLOCK_STRIDE(SH::THREADS)) {
    const int g = f % SH::G;
    const int it = f / SH::G;
    const int y0 = y0base + g;
    float2* rows = sm + g * SH::GSTRIDE;
    if (it == 0) {
      // kx = 0 and kx = M invert to real columns a, b: one inverse DFT of
      // A + i B gives a + i b (the imaginary parts of a and b, zero for a
      // Hermitian spectrum, are not separated)
      const int p0 = xp<SH>(0);
      {
        float2 xa[AY], xb[AY];
        load_col<SH>(xa, S, 0, z, y0, twny);
        load_col<SH>(xb, S, M, z, y0, twny);
#pragma unroll
        for (int k = 0; k < AY; ++k) xa[k] = make_float2(xa[k].x - xb[k].y, xa[k].y + xb[k].x);
        dft<AY, +1>(xa);
#pragma unroll
        for (int j = 0; j < AY; ++j)
          rows[j * RS + p0] = make_float2(xa[j].x + xa[j].y, xa[j].x - xa[j].y);
      }
      if constexpr (M % 2 == 0 && M >= 2) {
        float2 xh[AY];
        split_load<SH>(xh, S, M / 2, z, y0, twny);
        const int ph = xp<SH>(xrev<SH>(M / 2));
#pragma unroll
        for (int j = 0; j < AY; ++j) rows[j * RS + ph] = make_float2(2.f * xh[j].x, -2.f * xh[j].y);
      }
    } else {
      const int k = it;
      const int pa = xp<SH>(xrev<SH>(k));
      const int pb = xp<SH>(xrev<SH>(M - k));
      {
        float2 xc[AY];
        split_load<SH>(xc, S, k, z, y0, twny);
#pragma unroll
        for (int j = 0; j < AY; ++j) rows[j * RS + pa] = xc[j];
      }
      {
        float2 xc[AY];
        split_load<SH>(xc, S, M - k, z, y0, twny);
#pragma unroll
        for (int j = 0; j < AY; ++j) rows[j * RS + pb] = xc[j];
      }
      const float2 w = __ldg(&twr[k]);
#pragma unroll 4
      for (int j = 0; j < AY; ++j) {
        const float2 xa = rows[j * RS + pa];
        const float2 b = conjf2(rows[j * RS + pb]);
        const float2 e = cadd(xa, b);
        const float2 o = cmulc(csub(xa, b), w);
        rows[j * RS + pa] = make_float2(e.x - o.y, e.y + o.x);
        rows[j * RS + pb] = make_float2(e.x + o.y, -e.y + o.x);
      }
    }
  }
}

// ------------------------------------------------------------ Z tile passes
// y0 axis: lines (z, ki), element stride W; z axis: lines (y0, ki) = BW
// contiguous lines, element stride BW.
template <class SH, class A, int S, int DIR, bool ZAXIS>
__device__ __forceinline__ void z_tile_pass(float2* sm, const float2* __restrict__ tw) {
  constexpr int R = A::radix(S), len = A::len(S), span = len / R;
  constexpr int per_line = A::n / R, twstep = A::n / len;
  constexpr int nlines = ZAXIS ? SH::BW : SH::NZ * SH::W;
  constexpr int l0n = ZAXIS ? SH::BW : SH::W;       // lines adjacent in memory
  constexpr int es = ZAXIS ? SH::BW : SH::W;
  constexpr int s1 = ZAXIS ? 0 : SH::BW;
  constexpr int total = nlines * per_line;
#pragma unroll 1
  for (int f = threadIdx.x; f < total; f += CLARITY_BLOCK_STRIDE(SH::THREADS)) {
    const int l0 = f % l0n;
    const int rest = f / l0n;
    const int rem = rest % per_line;
    const int l1 = rest / per_line;
    const int b = rem / span;
    const int i = rem - b * span;
    const int base = l1 * s1 + l0 + (b * len + i) * es;
    float2 v[R];
#pragma unroll
    for (int t = 0; t < R; ++t) v[t] = sm[base + t * span * es];
    if constexpr (DIR < 0) {
      dft<R, -1>(v);
      if (span > 1 && i != 0) {
#pragma unroll
        for (int k = 1; k < R; ++k) v[k] = cmul(v[k], __ldg(&tw[i * k * twstep]));
      }
    } else {
      if (span > 1 && i != 0) {
#pragma unroll
        for (int k = 1; k < R; ++k) v[k] = cmulc(v[k], __ldg(&tw[i * k * twstep]));
      }
      dft<R, +1>(v);
    }
#pragma unroll
    for (int t = 0; t < R; ++t) sm[base + t * span * es] = v[t];
  }
}

template <class SH, class A, int S, bool ZAXIS>
__device__ __forceinline__ void tile_forward_from(float2* sm, const float2* tw) {
  if constexpr (S < A::npass) {
    z_tile_pass<SH, A, S, -1, ZAXIS>(sm, tw);
    __syncthreads();
    tile_forward_from<SH, A, S + 1, ZAXIS>(sm, tw);
  }
}
template <class SH, class A, int S, bool ZAXIS>
__device__ __forceinline__ void tile_inverse_down_to(float2* sm, const float2* tw) {
  if constexpr (S < A::npass) {
    tile_inverse_down_to<SH, A, S + 1, ZAXIS>(sm, tw);
    z_tile_pass<SH, A, S, +1, ZAXIS>(sm, tw);
    __syncthreads();
  }
}

// Last forward z pass, spectral operation, first inverse z pass: one
// register pass (the last DIF pass has span 1, so neither side needs
// twiddles).
template <class SH, class Mod>
__device__ __forceinline__ void z_mod_pass(float2* sm, const Mod& mod, long long gbase) {
  using A = typename SH::Z;
  constexpr int S = A::npass - 1;
  constexpr int R = A::radix(S);
  constexpr int nblk = A::n / R;
  constexpr int total = SH::BW * nblk;
  const Mod m = mod.resolved();
#pragma unroll 1
  for (int f = threadIdx.x; f < total; f += CLARITY_BLOCK_STRIDE(SH::THREADS)) {
    const int l0 = f % SH::BW;
    const int b = f / SH::BW;
    const int base = l0 + b * R * SH::BW;
    float2 v[R];
#pragma unroll
    for (int t = 0; t < R; ++t) v[t] = sm[base + t * SH::BW];
    dft<R, -1>(v);
#pragma unroll
    for (int t = 0; t < R; ++t) v[t] = m.apply(gbase + base + t * SH::BW, v[t]);
    dft<R, +1>(v);
#pragma unroll
    for (int t = 0; t < R; ++t) sm[base + t * SH::BW] = v[t];
  }
}

struct Tables {
  const float2* twx;   // w_M
  const float2* twy;   // w_By
  const float2* twz;   // w_nz
  const float2* twr;   // w_nx (r2c split)
  const float2* twny;  // w_ny (y split)
  int* err;            // device error word (bounded waits that gave up)
};

// ----------------------------------------------------------------- kernels
template <class SH, class Pro>
__global__ void __launch_bounds__(SH::THREADS, SH::XY_MINB)
    ks_xy_forward(const Pro pro, float2* __restrict__ S, const Tables T) {
  CLARITY_DYN_SMEM(float2, sm);
  const int z = blockIdx.x / SH::NGROUPS;
  const int y0base = (blockIdx.x - z * SH::NGROUPS) * SH::G;
  x_first<SH>(sm, pro, z, y0base, T.twx);
  __syncthreads();
  x_forward_from<SH, 1>(sm, T.twx);
  cols_forward<SH>(sm, S, z, y0base, T.twr, T.twny);
  pro.finish();
}

// Rows the epilogue reads are prefetched into L2 at kernel start, so their
// loads hit L2 by the time the transforms reach them.
template <class SH, class Epi>
__device__ __forceinline__ void prefetch_tile_rows(const Epi& epi, int z, int y0base) {
  if ((int)threadIdx.x < SH::ROWS) {
    const int r = threadIdx.x;
    const int g = r / SH::AY, j = r - g * SH::AY;
    epi.prefetch_row(y0base + g + SH::BY * j, z);
  }
}

template <class SH, class Epi>
__global__ void __launch_bounds__(SH::THREADS, SH::XY_MINB)
    ks_xy_inverse(Epi epi, const float2* __restrict__ S, const Tables T) {
  CLARITY_DYN_SMEM(float2, sm);
  const int z = blockIdx.x / SH::NGROUPS;
  const int y0base = (blockIdx.x - z * SH::NGROUPS) * SH::G;
  prefetch_tile_rows<SH>(epi, z, y0base);
  cols_inverse<SH>(sm, S, z, y0base, T.twr, T.twny);
  __syncthreads();
  x_inverse_down_to<SH, 1>(sm, T.twx);
  x_last<SH, Epi, false>(sm, epi, z, y0base, T.twx);
  epi.finish();
}

template <class SH, class Mid>
__global__ void __launch_bounds__(SH::THREADS, SH::XY_MINB)
    ks_xy_inv_fwd(Mid mid, float2* __restrict__ S, const Tables T) {
  CLARITY_DYN_SMEM(float2, sm);
  const int z = blockIdx.x / SH::NGROUPS;
  const int y0base = (blockIdx.x - z * SH::NGROUPS) * SH::G;
  // a plane whose result is known to be zero is neither read nor written;
  // the next Z pass reads those planes as zeros (Mod::zn)
  if (mid.zero_plane(z)) {  // neither read nor written (see Mod::zn)
    if constexpr (requires { mid.finish_skipped(); }) mid.finish_skipped();
    return;
  }
  prefetch_tile_rows<SH>(mid, z, y0base);
  const RowSkip<SH, Mid> skip{mid, z, y0base};
  cols_inverse<SH>(sm, S, z, y0base, T.twr, T.twny);
  __syncthreads();
  if constexpr (Mid::has_zero_rows) {
    // only rows j < L of each group can be nonzero; the others are zeroed
    const int L = mid.live_rows(y0base, SH::BY, SH::AY);
    x_inverse_down_to<SH, 1, RowSkip<SH, Mid>, true>(sm, T.twx, skip, L);
    x_last<SH, Mid, true, RowSkip<SH, Mid>, true>(sm, mid, z, y0base, T.twx, skip, L);
    const int dead = SH::G * (SH::AY - L) * SH::ROWSTRIDE;
    for (int t = threadIdx.x; t < dead; t += CLARITY_BLOCK_STRIDE(SH::THREADS)) {
      const int rd = t / SH::ROWSTRIDE, e = t - rd * SH::ROWSTRIDE;
      const int g = rd / (SH::AY - L), j = L + (rd - g * (SH::AY - L));
      sm[g * SH::GSTRIDE + j * SH::ROWSTRIDE + e] = make_float2(0.f, 0.f);
    }
    __syncthreads();
    x_forward_from<SH, 1, RowSkip<SH, Mid>, true>(sm, T.twx, skip, L);
  } else {
    x_inverse_down_to<SH, 1>(sm, T.twx, skip);
    x_last<SH, Mid, true>(sm, mid, z, y0base, T.twx, skip);
    __syncthreads();
    x_forward_from<SH, 1>(sm, T.twx, skip);
  }
  cols_forward<SH>(sm, S, z, y0base, T.twr, T.twny);
  mid.finish();
}

// First z stage of the spectral pass: the FP32 register pass, or (PREC > 0,
// a 16 x 16 z axis) its tensor-core form on split hi+lo operands.
template <class SH, int DIR, int PREC>
__device__ __forceinline__ void z_stage0(float2* sm, const float2* __restrict__ tw) {
#ifndef CLARITY_HOST_EMULATION
  if constexpr (PREC != kDftF32) {
    z_stage16_tc<SH, DIR, PREC>(sm, tw);
    return;
  }
#endif
  z_tile_pass<SH, typename SH::Z, 0, DIR, true>(sm, tw);
}

// Whether the tensor-core z stage applies to a shape: radix 16 first, whole
// groups of 8 lines, the tiled (not per-line) z kernel.
template <class SH>
constexpr bool kTcZ = SH::Z::radix(0) == 16 && SH::Z::npass >= 2 && SH::BW % 8 == 0 &&
                      !SH::Y_PER_LINE;

template <class SH, class Mod, int PREC = kDftF32>
__global__ void __launch_bounds__(SH::THREADS, SH::Z_MINB)
    ks_z(const Mod mod, const float2* __restrict__ Sin, float2* __restrict__ Sout,
         const Tables T) {
  CLARITY_DYN_SMEM(float2, sm);
  constexpr int tile = SH::TILE;
  const long long base = (long long)blockIdx.x * tile;
  if (threadIdx.x < 16) mod.prefetch_tile((unsigned)base, tile, threadIdx.x, 16);
  static_assert(tile % 2 == 0, "tile must be even");
  {
    // planes z >= zn are zero; BW is even so a float4 never spans two planes
    static_assert(SH::BW % 2 == 0, "tile rows must hold whole float4s");
    const int zn = mod.zn < SH::NZ ? mod.zn : SH::NZ;
    const int live4 = zn * SH::BW / 2;
    const float4* src = reinterpret_cast<const float4*>(Sin + base);
    float4* dst = reinterpret_cast<float4*>(sm);
#pragma unroll 4
    for (int t = threadIdx.x; t < tile / 2; t += CLARITY_BLOCK_STRIDE(SH::THREADS))
      dst[t] = t < live4 ? __ldg(&src[t]) : make_float4(0.f, 0.f, 0.f, 0.f);
  }
  __syncthreads();
  tile_forward_from<SH, typename SH::Y, 0, false>(sm, T.twy);
  if constexpr (Mod::forward_only) {
    tile_forward_from<SH, typename SH::Z, 0, true>(sm, T.twz);
  } else {
    // all z passes but the last, then last + spectral op + first inverse
    if constexpr (SH::Z::npass >= 2) {
      z_stage0<SH, -1, PREC>(sm, T.twz);
      __syncthreads();
    }
    if constexpr (SH::Z::npass >= 3) {
      z_tile_pass<SH, typename SH::Z, 1, -1, true>(sm, T.twz);
      __syncthreads();
    }
    z_mod_pass<SH>(sm, mod, base);
    __syncthreads();
    if constexpr (SH::Z::npass >= 3) {
      z_tile_pass<SH, typename SH::Z, 1, +1, true>(sm, T.twz);
      __syncthreads();
    }
    if constexpr (SH::Z::npass >= 2) {
      z_stage0<SH, +1, PREC>(sm, T.twz);
      __syncthreads();
    }
    tile_inverse_down_to<SH, typename SH::Y, 0, false>(sm, T.twy);
  }
  {
    // planes z >= zout are not needed downstream (BW even: whole float4s)
    const int zo = mod.zout < SH::NZ ? mod.zout : SH::NZ;
    const int out4 = zo * SH::BW / 2;
    float4* dst = reinterpret_cast<float4*>(Sout + base);
    const float4* src = reinterpret_cast<const float4*>(sm);
#pragma unroll 4
    for (int t = threadIdx.x; t < out4; t += CLARITY_BLOCK_STRIDE(SH::THREADS)) dst[t] = src[t];
  }
}

// ----------------------------------------------- Z kernel, y0 per line
// z-axis register pass S over the padded tile: lines l0 < BW (adjacent in
// memory), element e of line l0 at l0 + e*ZS.
template <class SH, int S, int DIR>
__device__ __forceinline__ void z2_pass(float2* sm, const float2* __restrict__ tw) {
  using A = typename SH::Z;
  constexpr int R = A::radix(S), len = A::len(S), span = len / R;
  constexpr int per_line = A::n / R, twstep = A::n / len;
  constexpr int total = SH::BW * per_line;
#pragma unroll 1
  for (int f = threadIdx.x; f < total; f += CLARITY_BLOCK_STRIDE(SH::THREADS)) {
    const int l0 = f % SH::BW;
    const int rem = f / SH::BW;
    const int b = rem / span;
    const int i = rem - b * span;
    const int base = l0 + (b * len + i) * SH::ZS;
    float2 v[R];
#pragma unroll
    for (int t = 0; t < R; ++t) v[t] = sm[base + t * span * SH::ZS];
    if constexpr (DIR < 0) {
      dft<R, -1>(v);
      if (span > 1 && i != 0) {
#pragma unroll
        for (int k = 1; k < R; ++k) v[k] = cmul(v[k], tw[i * k * twstep]);
      }
    } else {
      if (span > 1 && i != 0) {
#pragma unroll
        for (int k = 1; k < R; ++k) v[k] = cmulc(v[k], tw[i * k * twstep]);
      }
      dft<R, +1>(v);
    }
#pragma unroll
    for (int t = 0; t < R; ++t) sm[base + t * span * SH::ZS] = v[t];
  }
}

// Last z pass (span 1): forward DIF; then either the spectral operation and
// the first inverse pass back to smem, or (forward only) a store of the
// spectrum to HBM.  The global offset of tile element (z, l0) is
// gbase + z*BW + l0.
template <class SH, class Mod>
__device__ __forceinline__ void z2_last(float2* sm, const Mod& mod, unsigned gbase,
                                        float2* __restrict__ out) {
  using A = typename SH::Z;
  constexpr int S = A::npass - 1;
  constexpr int R = A::radix(S);
  constexpr int nblk = A::n / R;
  constexpr int total = SH::BW * nblk;
  const Mod m = mod.resolved();
#pragma unroll 1
  for (int f = threadIdx.x; f < total; f += CLARITY_BLOCK_STRIDE(SH::THREADS)) {
    const int l0 = f % SH::BW;
    const int b = f / SH::BW;
    const int sbase = l0 + b * R * SH::ZS;
    const unsigned g0 = gbase + l0 + b * R * SH::BW;
    float2 v[R];
#pragma unroll
    for (int t = 0; t < R; ++t) v[t] = sm[sbase + t * SH::ZS];
    dft<R, -1>(v);
    if constexpr (Mod::forward_only) {
#pragma unroll
      for (int t = 0; t < R; ++t) out[g0 + t * SH::BW] = v[t];
    } else {
#pragma unroll
      for (int t = 0; t < R; ++t) v[t] = m.apply(g0 + t * SH::BW, v[t]);
      dft<R, +1>(v);
#pragma unroll
      for (int t = 0; t < R; ++t) sm[sbase + t * SH::ZS] = v[t];
    }
  }
}

template <class SH, class Mod>
__global__ void __launch_bounds__(SH::THREADS, SH::Z_MINB)
    ks_z2(const Mod mod, const float2* __restrict__ Sin, float2* __restrict__ Sout,
          const Tables T) {
  CLARITY_PDL_WAIT();  // the previous kernel's output is complete and visible
  CLARITY_DYN_SMEM(float2, sm);
  static_assert(SH::Y_PER_LINE, "y0 per-line Z kernel needs BY <= 32");
  constexpr int BY = SH::BY, W = SH::W, BW = SH::BW, NZ = SH::NZ, ZS = SH::ZS;
  // z rows of the tile are contiguous BW*8-byte runs in HBM and land at
  // ZS*8-byte strides in shared memory: bulk copies when both are 16-byte
  // multiples
  constexpr bool BULK = (BW * 8) % 16 == 0 && (ZS * 8) % 16 == 0;
  using A = typename SH::Z;
  const unsigned gbase = blockIdx.x * (unsigned)SH::TILE;
  const int zn = mod.zn < NZ ? mod.zn : NZ;  // planes z >= zn are zero
  if (threadIdx.x < 16) mod.prefetch_tile(gbase, SH::TILE, threadIdx.x, 16);
  // z twiddles in shared memory: a z-pass task's twiddle is the same for all
  // lanes of a warp (a broadcast), where the table in global memory cost an
  // L1 round trip per twiddle
  float2* twz = sm + SH::Z2_TILE_BYTES / 8;
  for (int t = threadIdx.x; t < NZ; t += CLARITY_BLOCK_STRIDE(SH::THREADS)) twz[t] = __ldg(&T.twz[t]);
  __shared__ alignas(8) uint64_t bar;
  if constexpr (BULK) {
    static_assert((BW * 8) % 16 == 0 && (ZS * 8) % 16 == 0 && (SH::TILE * 8) % 16 == 0,
                  "bulk copies need 16-byte sizes and offsets");
    if (!smem_aligned16(sm)) {  // never expected: refuse rather than fault
      if (threadIdx.x == 0) raise_error(T.err, kErrMisaligned);
      return;
    }
    if (threadIdx.x == 0) mbar_init(&bar, 1);
    __syncthreads();
    if ((int)threadIdx.x < CLARITY_ISSUE_LANES) {
      if (threadIdx.x == 0) mbar_arrive_expect_tx(&bar, (uint32_t)(zn * BW * 8));
      __syncwarp();
      for (int z = threadIdx.x; z < zn; z += CLARITY_ISSUE_LANES)
        bulk_load(sm + z * ZS, Sin + gbase + z * BW, BW * 8, &bar);
    }
    if (!mbar_wait(&bar, 0, T.err)) {
      mbar_wait(&bar, 0, nullptr);  // give copies in flight a last chance
      return;
    }
  }
  // y0 forward, one line (z, ki) per thread
#pragma unroll 1
  for (int l = threadIdx.x; l < NZ * W; l += CLARITY_BLOCK_STRIDE(SH::THREADS)) {
    const int ki = l % W, z = l / W;
    float2 v[BY];
    float2* d = sm + z * ZS + ki;
    if (z >= zn) {  // known-zero plane: its transform is zero
#pragma unroll
      for (int k = 0; k < BY; ++k) d[k * W] = make_float2(0.f, 0.f);
      continue;
    }
    if constexpr (BULK) {
#pragma unroll
      for (int y = 0; y < BY; ++y) v[y] = d[y * W];
    } else {
      const float2* src = Sin + gbase + z * BW + ki;
#pragma unroll
      for (int y = 0; y < BY; ++y) v[y] = __ldg(&src[y * W]);
    }
    dft<BY, -1>(v);
#pragma unroll
    for (int k = 0; k < BY; ++k) d[k * W] = v[k];
  }
  __syncthreads();
  if constexpr (A::npass >= 2) {
    z2_pass<SH, 0, -1>(sm, twz);
    __syncthreads();
  }
  if constexpr (A::npass >= 3) {
    z2_pass<SH, 1, -1>(sm, twz);
    __syncthreads();
  }
  z2_last<SH>(sm, mod, gbase, Sout);
  if constexpr (!Mod::forward_only) {
    __syncthreads();
    if constexpr (A::npass >= 3) {
      z2_pass<SH, 1, +1>(sm, twz);
      __syncthreads();
    }
    if constexpr (A::npass >= 2) {
      z2_pass<SH, 0, +1>(sm, twz);
      __syncthreads();
    }
    // y0 inverse per line, for the planes the next pass reads (z < zo)
    const int zo = mod.zout < NZ ? mod.zout : NZ;
#pragma unroll 1
    for (int l = threadIdx.x; l < zo * W; l += CLARITY_BLOCK_STRIDE(SH::THREADS)) {
      const int ki = l % W, z = l / W;
      float2* d = sm + z * ZS + ki;
      float2 v[BY];
#pragma unroll
      for (int k = 0; k < BY; ++k) v[k] = d[k * W];
      dft<BY, +1>(v);
      if constexpr (BULK) {
#pragma unroll
        for (int y = 0; y < BY; ++y) d[y * W] = v[y];
      } else {
        float2* dst = Sout + gbase + z * BW + ki;
#pragma unroll
        for (int y = 0; y < BY; ++y) dst[y * W] = v[y];
      }
    }
    if constexpr (BULK) {
      fence_smem_to_async();
      __syncthreads();
      if ((int)threadIdx.x < CLARITY_ISSUE_LANES) {
        for (int z = threadIdx.x; z < zo; z += CLARITY_ISSUE_LANES)
          bulk_store(Sout + gbase + z * BW, sm + z * ZS, BW * 8);
        bulk_store_commit_and_wait();
      }
    }
  }
}

// Does a runtime plan match shape SH exactly (same radices and tiling)?
template <class SH>
inline bool matches(const VolPlan& P) {
  auto same_axis = [](const AxisPlan& A, auto rad) {
    using R = decltype(rad);
    if (A.n != R::n || A.npass != R::npass) return false;
    for (int s = 0; s < A.npass; ++s)
      if (A.radix[s] != R::radix(s)) return false;
    return true;
  };
  return P.xmode == 0 && P.M == SH::M && P.Ay == SH::AY && P.By == SH::BY &&
         P.nz == SH::NZ && P.G == SH::G && P.W == SH::W && P.rowStride == SH::ROWSTRIDE &&
         P.padShift == SH::PADSHIFT && same_axis(P.ax, typename SH::X{}) &&
         same_axis(P.ayB, typename SH::Y{}) && same_axis(P.az, typename SH::Z{});
}

}  // namespace st
}  // namespace clarity
