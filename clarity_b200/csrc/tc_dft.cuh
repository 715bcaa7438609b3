// tc_dft.cuh -- the first radix-16 stage of the z axis as tensor-core GEMMs on
// split hi+lo operands (the precision form of the 3-D FFT).
//
// A radix-16 DIF stage applies the 16-point DFT to every line of the stage:
// Y = F16 X with X one column per line.  In real arithmetic that is
//     [Yr]   [Fr  -Fi] [Xr]
//     [Yi] = [Fi   Fr] [Xi],
// a 32x32 matrix times 32 x (lines) -- two m-tiles by two k-steps of
// mma.sync.m16n8k16 per 8 lines.  Operands are split into a high and a low
// part of the 16-bit type (x = hi + lo, lo = x - hi rounded again), and the
// product is hi*hi + hi*lo + lo*hi with FP32 accumulation (the lo*lo term is
// below FP32 resolution for FP16 and is dropped for both types):
//   * FP16: 11 + 11 significant bits -- FP32-class accuracy.  FP16's range is
//     small, so each warp's 8-line tile is scaled by a power of two that
//     brings its largest magnitude just below 2^15 and unscaled after the MMA.
//   * BF16: 8 + 8 bits, FP32's range (no scaling) -- about 2^-16 relative.
// The twiddles of the stage (w_n^(i k), the DIF span factors) stay in FP32
// on the CUDA cores.  The stage replaces the SIMT register pass it mirrors
// (z_tile_pass, stage 0) in the specialised z kernel when the library's DFT
// precision mode asks for it; every other pass is unchanged.
#pragma once
#include <cstdint>

#include "dft_codelets.cuh"
#include "launch_macro.cuh"

#ifndef CLARITY_HOST_EMULATION
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#endif

namespace clarity {
namespace st {

// The library's DFT precision modes (clarityx_set_dft_precision).
enum DftPrecision { kDftF32 = 0, kDftF16Split = 1, kDftBF16Split = 2 };

#ifndef CLARITY_HOST_EMULATION
template <int PREC>
struct TcType;

template <>
struct TcType<kDftF16Split> {
  static constexpr bool kScaled = true;
  static __device__ __forceinline__ uint32_t pack(float a, float b) {
    const __half2 h = __floats2half2_rn(a, b);
    return *reinterpret_cast<const uint32_t*>(&h);
  }
  static __device__ __forceinline__ float2 unpack(uint32_t u) {
    return __half22float2(*reinterpret_cast<const __half2*>(&u));
  }
  static __device__ __forceinline__ void mma(float (&d)[4], const uint32_t (&a)[4], uint32_t b0,
                                             uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 "
        "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
  }
};

template <>
struct TcType<kDftBF16Split> {
  static constexpr bool kScaled = false;
  static __device__ __forceinline__ uint32_t pack(float a, float b) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const uint32_t*>(&h);
  }
  static __device__ __forceinline__ float2 unpack(uint32_t u) {
    return __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&u));
  }
  static __device__ __forceinline__ void mma(float (&d)[4], const uint32_t (&a)[4], uint32_t b0,
                                             uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
        "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
  }
};

// (a, b) -> packed hi pair and packed lo pair: hi = T(a), lo = T(a - hi).
template <int PREC>
__device__ __forceinline__ void split2(float a, float b, uint32_t& hi, uint32_t& lo) {
  hi = TcType<PREC>::pack(a, b);
  const float2 h = TcType<PREC>::unpack(hi);
  lo = TcType<PREC>::pack(a - h.x, b - h.y);
}

// Stage 0 of the z axis (radix 16, span n/16) over the tile, forward DIF
// (DIR -1: DFT, then v[k] *= w_n^(i k)) or inverse DIT (DIR +1: v[t] *=
// conj(w_n^(i t)), then the unnormalised inverse DFT), exactly as
// z_tile_pass<SH, Z, 0, DIR, true> computes it in FP32.  Element t of line
// (l0, i) sits at sm[l0 + (i + span t) BW].  One warp takes 8 lines of the
// same i at a time: mma fragment column n = line l0base + n, k rows = t for
// the input and the output frequency for the result.
template <class SH, int DIR, int PREC>
__device__ __forceinline__ void z_stage16_tc(float2* sm, const float2* __restrict__ tw) {
  using A = typename SH::Z;
  static_assert(A::radix(0) == 16 && A::npass >= 2, "stage 0 must be radix 16");
  static_assert(SH::BW % 8 == 0, "lines come in groups of 8");
  constexpr int span = A::n / 16;
  constexpr int es = SH::BW;
  constexpr int NB = SH::BW / 8;
  constexpr int ntiles = span * NB;
  constexpr int nwarps = SH::THREADS / 32;
  using T = TcType<PREC>;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, c = lane & 3;
  // A fragments of F[k][t] = exp(DIR 2 pi i k t / 16): register r holds
  // rows {g, g+8, g, g+8}[r], columns {2c, 2c, 2c+8, 2c+8}[r] + (0, 1).
  // Entries from FP64 sincospi, rounded to float, then split.
  uint32_t frh[4], frl[4], fih[4], fil[4], nfih[4], nfil[4];
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const int row = (r & 1) ? g + 8 : g;
    const int col = (r & 2) ? 2 * c + 8 : 2 * c;
    float re[2], im[2];
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const int kt = (row * (col + q)) & 15;
      double s, co;
      sincospi((double)kt / 8.0, &s, &co);
      re[q] = (float)co;
      im[q] = (float)(DIR * s);
    }
    split2<PREC>(re[0], re[1], frh[r], frl[r]);
    split2<PREC>(im[0], im[1], fih[r], fil[r]);
    split2<PREC>(-im[0], -im[1], nfih[r], nfil[r]);
  }
#pragma unroll 1
  for (int nt = warp; nt < ntiles; nt += nwarps) {
    const int i = nt / NB;
    const int lbase = (nt - i * NB) * 8;
    // this lane's inputs: line lbase + g, t = 2c, 2c+1, 2c+8, 2c+9
    float2 x[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int t = 2 * c + (q & 1) + ((q & 2) ? 8 : 0);
      x[q] = sm[lbase + g + (i + span * t) * es];
      if (DIR > 0 && i != 0) x[q] = cmulc(x[q], __ldg(&tw[i * t]));
    }
    float s = 1.f, inv = 1.f;
    if constexpr (T::kScaled) {
      float m = 0.f;
#pragma unroll
      for (int q = 0; q < 4; ++q) m = fmaxf(m, fmaxf(fabsf(x[q].x), fabsf(x[q].y)));
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
      int e = 0;
      frexpf(m, &e);  // m < 2^e
      s = ldexpf(1.f, 15 - e);
      inv = ldexpf(1.f, e - 15);
    }
    uint32_t rh0, rl0, rh1, rl1, ih0, il0, ih1, il1;
    split2<PREC>(x[0].x * s, x[1].x * s, rh0, rl0);  // k rows 2c, 2c+1
    split2<PREC>(x[2].x * s, x[3].x * s, rh1, rl1);  // k rows 2c+8, 2c+9
    split2<PREC>(x[0].y * s, x[1].y * s, ih0, il0);
    split2<PREC>(x[2].y * s, x[3].y * s, ih1, il1);
    float dr[4] = {0.f, 0.f, 0.f, 0.f}, di[4] = {0.f, 0.f, 0.f, 0.f};
    // Yr = Fr Xr - Fi Xi, Yi = Fi Xr + Fr Xi; the small cross terms first
    T::mma(dr, frl, rh0, rh1);
    T::mma(dr, frh, rl0, rl1);
    T::mma(dr, nfil, ih0, ih1);
    T::mma(dr, nfih, il0, il1);
    T::mma(dr, frh, rh0, rh1);
    T::mma(dr, nfih, ih0, ih1);
    T::mma(di, fil, rh0, rh1);
    T::mma(di, fih, rl0, rl1);
    T::mma(di, frl, ih0, ih1);
    T::mma(di, frh, il0, il1);
    T::mma(di, fih, rh0, rh1);
    T::mma(di, frh, ih0, ih1);
    __syncwarp();
    // result fragment: (row k, column line) = (g, 2c + q) for q < 2,
    // (g + 8, 2c + q - 2) for q >= 2
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int k = q < 2 ? g : g + 8;
      const int line = lbase + 2 * c + (q & 1);
      float2 y = make_float2(dr[q] * inv, di[q] * inv);
      if (DIR < 0 && i != 0) y = cmul(y, __ldg(&tw[i * k]));
      sm[line + (i + span * k) * es] = y;
    }
  }
}
#endif

}  // namespace st
}  // namespace clarity
