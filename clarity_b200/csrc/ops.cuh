// ops.cuh -- operations fused into the FFT passes.
//
// Prologues (XY forward): load_c(m, y, z) returns complex row element m of
//   row (y, z): (v[2m], v[2m+1]) for even nx, (v[m], 0) for odd nx.
// Epilogues (XY inverse): apply_c(m, y, z, c) receives the same pair of
//   real-space values after the inverse transform; the returned pair feeds
//   the forward transform when the epilogue is fused into k_xy_inv_fwd.
// Spectral operations (Z pass): apply(idx, v) with idx the element's offset
//   in the S layout (the OTF shares that layout).
#pragma once
#include "launch_macro.cuh"

#include "dft_codelets.cuh"
#include "plan.hpp"
#include "tma.cuh"

namespace clarity {
namespace st {
// A tile row's input for the staged pass kernels: nf floats at p
// (x = 0 .. nf-1), zero beyond; nf == 0 for a row known to be zero.
struct RowRef {
  const float* p;
  int nf;
};
}  // namespace st

// The reference divide of src/ComputePrimitives.cxx:144-148 (and
// ComputePrimitivesGPU.cu:180-184) tests fabs(b) < 1e-5 in double; for a
// float b that is exactly fabsf(b) <= 1e-5f (1e-5f is the largest float
// below 1e-5).
__device__ __forceinline__ float rl_ratio(float g, float b) {
  return (fabsf(b) <= 1e-5f) ? 0.f : g / b;
}

// Real volume on the padded work box, x fastest.  The planner rejects boxes
// of 2^31 voxels or more, so 32-bit offsets suffice.
struct WorkVol {
  int nx, ny, nz;
  __device__ __forceinline__ unsigned idx(int x, int y, int z) const {
    return ((unsigned)z * ny + y) * nx + x;
  }
};

// Unpadded image seen on the work box with zero shift
// (src/MaximumLikelihoodDeconvolve.cxx:278-282): the image itself inside
// [0,X)x[0,Y)x[0,Z), zero in the padding.  Only bounds checks, no modulo.
struct ImageSrc {
  const float* CLARITY_RESTRICT src;
  int X, Y, Z;
  __device__ __forceinline__ float at(int x, int y, int z) const {
    if (x < X && y < Y && z < Z) return CLARITY_LDG(&src[((unsigned)z * Y + y) * X + x]);
    return 0.f;
  }
};

// Source volume of size (X, Y, Z) seen on the work box through the
// reference's cyclic pad/shift (src/ImagePadSpatialShift.cxx:42-66):
// work coordinate d maps to s = ((d - shift) wrapped) % dim, inside when
// s < src dim, otherwise the fill value (0).
struct PaddedSrc {
  const float* CLARITY_RESTRICT src;
  int X, Y, Z;       // source dims
  int sx, sy, sz;    // shift
  int nx, ny, nz;    // work dims
  __device__ __forceinline__ static int wrap(int d, int shift, int n) {
    int s = d - shift;
    if (s < 0) s += n;
    return s % n;
  }
  __device__ __forceinline__ float at(int x, int y, int z) const {
    const int k = wrap(z, sz, nz);
    const int j = wrap(y, sy, ny);
    const int i = wrap(x, sx, nx);
    if (i >= 0 && j >= 0 && k >= 0 && i < X && j < Y && k < Z)
      return CLARITY_LDG(&src[((long long)k * Y + j) * X + i]);
    return 0.f;
  }
};

// ---------------------------------------------------------------- prologues
// Plain work-box volume, optionally multiplied by a device-resident scale
// (the deferred RL flux rescale).
struct ProWork {
  const float* CLARITY_RESTRICT v;
  const float* CLARITY_RESTRICT scale;  // nullptr -> 1
  WorkVol w;
  int xmode;
  __device__ __forceinline__ float2 load_c(int m, int y, int z) const {
    const float s = scale ? *scale : 1.f;
    if (xmode == 0) {
      const float2 a = CLARITY_LDG(reinterpret_cast<const float2*>(v + w.idx(2 * m, y, z)));
      return scale ? make_float2(s * a.x, s * a.y) : a;
    }
    const float a = CLARITY_LDG(&v[w.idx(m, y, z)]);
    return make_float2(scale ? s * a : a, 0.f);
  }
  __device__ __forceinline__ void finish() const {}
};

// Extrapolated estimate of accelerated RL (Biggs-Andrews): y = max(0,
// x + alpha (x - xp)), one fused multiply-add, stored to yout on the way into
// the forward transform (the product step reads it back as the estimate).
struct ProAccel {
  const float* CLARITY_RESTRICT x;
  const float* CLARITY_RESTRICT xp;
  const float* CLARITY_RESTRICT alpha;
  float* CLARITY_RESTRICT yout;
  WorkVol w;
  int xmode;
  __device__ __forceinline__ static float extrap(float a, float x, float xp) {
    return fmaxf(0.f, fmaf(a, x - xp, x));
  }
  __device__ __forceinline__ float2 load_c(int m, int y, int z) const {
    const float a = CLARITY_LDG(alpha);
    if (xmode == 0) {
      const unsigned i = w.idx(2 * m, y, z);
      const float2 xv = CLARITY_LDG(reinterpret_cast<const float2*>(x + i));
      const float2 pv = CLARITY_LDG(reinterpret_cast<const float2*>(xp + i));
      const float2 r = make_float2(extrap(a, xv.x, pv.x), extrap(a, xv.y, pv.y));
      *reinterpret_cast<float2*>(yout + i) = r;
      return r;
    }
    const unsigned i = w.idx(m, y, z);
    const float r = extrap(a, CLARITY_LDG(x + i), CLARITY_LDG(xp + i));
    yout[i] = r;
    return make_float2(r, 0.f);
  }
  __device__ __forceinline__ void finish() const {}
};

// Unpadded source read through the pad/shift map, times an optional scale.
struct ProPadded {
  PaddedSrc p;
  const float* CLARITY_RESTRICT scale;  // nullptr -> 1
  int xmode;
  __device__ __forceinline__ float2 load_c(int m, int y, int z) const {
    const float s = scale ? *scale : 1.f;
    if (xmode == 0) {
      float a = p.at(2 * m, y, z), b = p.at(2 * m + 1, y, z);
      if (scale) { a = s * a; b = s * b; }
      return make_float2(a, b);
    }
    float a = p.at(m, y, z);
    if (scale) a = s * a;
    return make_float2(a, 0.f);
  }
  __device__ __forceinline__ void finish() const {}
};

// The padded image (zero shift) as a prologue.
struct ProImage {
  ImageSrc p;
  int xmode;
  __device__ __forceinline__ float2 load_c(int m, int y, int z) const {
    if (xmode == 0) return make_float2(p.at(2 * m, y, z), p.at(2 * m + 1, y, z));
    return make_float2(p.at(m, y, z), 0.f);
  }
  __device__ __forceinline__ void finish() const {}
};

// ---------------------------------------------------------------- epilogues
// Block-wide FP64 sum of per-thread partials into partial[block index]
// (fixed reduction order: deterministic).
__device__ __forceinline__ void block_sum_store(double acc, double* partial) {
  __shared__ double red[32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) red[warp] = acc;
  __syncthreads();
  if (warp == 0) {
    const int nw = (blockDim.x + 31) >> 5;
    double a = lane < nw ? red[lane] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    if (lane == 0) partial[CLARITY_BLOCK_ID()] = a;
  }
}

// Block-wide FP64 total of np partials (thread 0 gets it; fixed order):
// thread i sums partials i, i + blockDim.x, ..., then a tree over the block.
// The partials are read through L2 (__ldcg); they come from the previous
// kernel on the stream.
__device__ __forceinline__ double block_total(const double* partial, int np) {
  double acc = 0;
  for (int i = threadIdx.x; i < np; i += blockDim.x) acc += __ldcg(&partial[i]);
  __shared__ double red[32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) red[warp] = acc;
  __syncthreads();
  double t = 0;
  if (threadIdx.x == 0) {
    for (int w = 0; w < (int)((blockDim.x + 31) >> 5); ++w) t += red[w];
  }
  return t;  // valid in thread 0
}

// Store the real-space result on the work box.
struct EpiWork {
  static constexpr bool has_zero_rows = false;
  float* CLARITY_RESTRICT out;
  WorkVol w;
  int xmode;
  __device__ __forceinline__ float2 apply_c(int m, int y, int z, float2 c) {
    if (xmode == 0)
      *reinterpret_cast<float2*>(out + w.idx(2 * m, y, z)) = c;
    else
      out[w.idx(m, y, z)] = c.x;
    return c;
  }
    // padding rows / z planes where the result is known to be zero
  __device__ __forceinline__ bool zero_row(int, int) const { return false; }
  __device__ __forceinline__ bool zero_plane(int) const { return false; }
  // rows y0base + BY*j, j < live_rows, can be nonzero (all here)
  __device__ __forceinline__ int live_rows(int, int, int ay) const { return ay; }
  __device__ __forceinline__ void prefetch_row(int, int) const {}
  __device__ __forceinline__ void finish() {}
};

// Store only the image region (crop from the origin, src/ImageClip.cxx:41-46)
// into an unpadded (X, Y, Z) volume, times an optional device scale.
struct EpiClip {
  static constexpr bool has_zero_rows = false;
  float* CLARITY_RESTRICT out;
  int X, Y, Z;
  const float* CLARITY_RESTRICT scale;
  int xmode;
  __device__ __forceinline__ void put(int x, int y, int z, float v) {
    if (x < X && y < Y && z < Z) {
      if (scale) v = *scale * v;
      out[((long long)z * Y + y) * X + x] = v;
    }
  }
  __device__ __forceinline__ float2 apply_c(int m, int y, int z, float2 c) {
    if (xmode == 0) {
      put(2 * m, y, z, c.x);
      put(2 * m + 1, y, z, c.y);
    } else {
      put(m, y, z, c.x);
    }
    return c;
  }
    // padding rows / z planes where the result is known to be zero
  __device__ __forceinline__ bool zero_row(int, int) const { return false; }
  __device__ __forceinline__ bool zero_plane(int) const { return false; }
  // rows y0base + BY*j, j < live_rows, can be nonzero (all here)
  __device__ __forceinline__ int live_rows(int, int, int ay) const { return ay; }
  __device__ __forceinline__ void prefetch_row(int, int) const {}
  __device__ __forceinline__ void finish() {}
};

// RL step 4 (src/MaximumLikelihoodDeconvolve.cxx:69-70) with the flux sum of
// step 5 (:73-74): u_new = cur * c, cur = scale * u (or the padded image on
// the first iteration), partial sums of u_new in FP64.
struct EpiRLProduct {
  static constexpr bool has_zero_rows = false;
  static constexpr int kFamily = KK_XY_PRODUCT;
  const float* CLARITY_RESTRICT cur;     // work-box estimate, or nullptr
  ImageSrc g;                        // used when cur == nullptr
  const float* CLARITY_RESTRICT scale;   // deferred flux scale for cur
  float* CLARITY_RESTRICT unew;
  double* CLARITY_RESTRICT partial;
  WorkVol w;
  int xmode;
  double acc;
  int* nblocks = nullptr;  // receives the grid size (the number of partials), or nullptr
  __device__ __forceinline__ float cur_at(int x, int y, int z) const {
    if (cur) {
      const float u = CLARITY_LDG(&cur[w.idx(x, y, z)]);
      return scale ? *scale * u : u;
    }
    return g.at(x, y, z);
  }
  __device__ __forceinline__ float2 apply_c(int m, int y, int z, float2 c) {
    if (xmode == 0) {
      const float a = cur_at(2 * m, y, z) * c.x;
      const float b = cur_at(2 * m + 1, y, z) * c.y;
      *reinterpret_cast<float2*>(unew + w.idx(2 * m, y, z)) = make_float2(a, b);
      acc += (double)a;
      acc += (double)b;
      return make_float2(a, b);
    }
    const float a = cur_at(m, y, z) * c.x;
    unew[w.idx(m, y, z)] = a;
    acc += (double)a;
    return make_float2(a, 0.f);
  }
    // padding rows / z planes where the result is known to be zero
  __device__ __forceinline__ bool zero_row(int, int) const { return false; }
  __device__ __forceinline__ bool zero_plane(int) const { return false; }
  // rows y0base + BY*j, j < live_rows, can be nonzero (all here)
  __device__ __forceinline__ int live_rows(int, int, int ay) const { return ay; }
  // the estimate row this block's epilogue will read, into L2
  __device__ __forceinline__ void prefetch_row(int y, int z) const {
    if (cur) prefetch_l2_range(cur + w.idx(0, y, z), sizeof(float) * (size_t)w.nx);
  }
  // Staged form (passes_xy_tma.cuh): row (y, z) of cur (or of the image on
  // the first iteration) arrives in shared memory; u' overwrites it there and
  // leaves by a bulk store to unew.
  static constexpr bool kStaged = true;
  static constexpr bool kStoreRows = true;
  __device__ __forceinline__ st::RowRef in_row(int y, int z) const {
    if (cur) return {cur + w.idx(0, y, z), w.nx};
    if (y < g.Y && z < g.Z) return {g.src + ((unsigned)z * g.Y + y) * g.X, g.X};
    return {nullptr, 0};
  }
  __device__ __forceinline__ float* out_row(int y, int z) const { return unew + w.idx(0, y, z); }
  __device__ __forceinline__ float2 apply_s(int m, int, int, float2 c, float* sr, int n) {
    const int x = 2 * m;
    float u0 = x < n ? sr[x] : 0.f, u1 = x + 1 < n ? sr[x + 1] : 0.f;
    if (cur && scale) {
      const float s = CLARITY_LDG(scale);
      u0 = s * u0;
      u1 = s * u1;
    }
    const float a = u0 * c.x, b = u1 * c.y;
    sr[x] = a;
    sr[x + 1] = b;
    acc += (double)a;
    acc += (double)b;
    return make_float2(a, b);
  }
  __device__ __forceinline__ void finish() {
    block_sum_store(acc, partial);
    if (nblocks && CLARITY_BLOCK_ID() == 0 && threadIdx.x == 0) *nblocks = (int)CLARITY_GRID_DIM();
  }
};

// RL step 2 (src/MaximumLikelihoodDeconvolve.cxx:61-62): r = g / (h*u) with
// the 1e-5 guard, fused between the inverse and forward transforms.
struct MidRLRatio {
  static constexpr bool has_zero_rows = true;
  ImageSrc g;
  int xmode;
  // Optional trace (idiv_partial != nullptr): the I-divergence of g against
  // b = h*cur over the image, g ln(g/b) + b - g with 0 ln 0 = 0 (terms with
  // g > 0 >= b skipped), summed in FP64 per block; block 0 stores the grid
  // size in *nblocks.  Same definition as k_idiv and the oracle
  // (IDIVFunctional, src/IDivergenceDeconvolve.cxx:33-47, alpha = 0).
  double* CLARITY_RESTRICT idiv_partial = nullptr;
  int* nblocks = nullptr;
  double acc = 0.0;
  __device__ __forceinline__ void idiv_add(float a, float b) {
    if (a > 0.f) {
      if (b > 0.f) {
        const double da = a, db = b;
        acc += da * log(da / db) + db - da;
      }
    } else {
      acc += (double)b - (double)a;
    }
  }
  __device__ __forceinline__ float2 apply_c(int m, int y, int z, float2 b) {
    if (idiv_partial && y < g.Y && z < g.Z) {
      if (xmode == 0) {
        if (2 * m < g.X) idiv_add(g.at(2 * m, y, z), b.x);
        if (2 * m + 1 < g.X) idiv_add(g.at(2 * m + 1, y, z), b.y);
      } else if (m < g.X) {
        idiv_add(g.at(m, y, z), b.x);
      }
    }
    if (xmode == 0)
      return make_float2(rl_ratio(g.at(2 * m, y, z), b.x),
                         rl_ratio(g.at(2 * m + 1, y, z), b.y));
    return make_float2(rl_ratio(g.at(m, y, z), b.x), 0.f);
  }
    // g is zero outside the image, so the ratio is exactly zero there
  // (0/b, or the 1e-5 guard): rows with y >= Y and planes with z >= Z need no
  // transform at all
  __device__ __forceinline__ bool zero_row(int y, int z) const { return y >= g.Y || z >= g.Z; }
  __device__ __forceinline__ bool zero_plane(int z) const { return z >= g.Z; }
  // planes a launch needs to cover (the rest are zero_plane)
  int live_planes(int nz) const { return g.Z < nz ? g.Z : nz; }
  // rows y0base + by*j with j < live_rows lie inside the image (y < Y)
  __device__ __forceinline__ int live_rows(int y0base, int by, int ay) const {
    const int l = (g.Y - y0base + by - 1) / by;
    return l < 0 ? 0 : (l > ay ? ay : l);
  }
  __device__ __forceinline__ void prefetch_row(int y, int z) const {
    if (y < g.Y && z < g.Z)
      prefetch_l2_range(g.src + ((unsigned)z * g.Y + y) * g.X, sizeof(float) * (size_t)g.X);
  }
  // Staged form: the image row arrives in shared memory.
  static constexpr bool kStaged = true;
  static constexpr bool kStoreRows = false;
  __device__ __forceinline__ st::RowRef in_row(int y, int z) const {
    if (y < g.Y && z < g.Z) return {g.src + ((unsigned)z * g.Y + y) * g.X, g.X};
    return {nullptr, 0};
  }
  __device__ __forceinline__ float* out_row(int, int) const { return nullptr; }
  __device__ __forceinline__ float2 apply_s(int m, int, int, float2 b, float* sr, int n) {
    const int x = 2 * m;
    const float a0 = x < n ? sr[x] : 0.f, a1 = x + 1 < n ? sr[x + 1] : 0.f;
    if (idiv_partial) {
      if (x < n) idiv_add(a0, b.x);
      if (x + 1 < n) idiv_add(a1, b.y);
    }
    return make_float2(rl_ratio(a0, b.x), rl_ratio(a1, b.y));
  }
  __device__ __forceinline__ void finish() {
    if (idiv_partial) {
      block_sum_store(acc, idiv_partial);
      if (nblocks && CLARITY_BLOCK_ID() == 0 && threadIdx.x == 0) *nblocks = (int)CLARITY_GRID_DIM();
    }
  }
  // a block that returned early (plane outside the image) contributes zero
  __device__ __forceinline__ void finish_skipped() {
    if (idiv_partial && threadIdx.x == 0) {
      idiv_partial[CLARITY_BLOCK_ID()] = 0.0;
      if (nblocks && CLARITY_BLOCK_ID() == 0) *nblocks = (int)CLARITY_GRID_DIM();
    }
  }
};

// JVC update (src/JansenVanCittertDeconvolve.cxx:106-111,
// JansenVanCittertDeconvolveGPU.cu:43-49): i' = max(0, i + gamma(o) (g - o)),
// gamma(o) = 1 - (o - A)^2 / A^2.  cur == nullptr reads i from the padded
// image (first update).  Stores i' on the work box and returns it, so the
// fused kernel transforms it for the next iteration.
struct EpiJVC {
  static constexpr bool has_zero_rows = false;
  const float* CLARITY_RESTRICT cur;
  ImageSrc g;
  float* CLARITY_RESTRICT inext;
  float A, invASq;
  WorkVol w;
  int xmode;
  __device__ __forceinline__ float upd(float i, float gv, float o) const {
    const float diff = o - A;
    const float gamma = 1.0f - ((diff * diff) * invASq);
    const float val = i + (gamma * (gv - o));
    return val < 0.0f ? 0.0f : val;
  }
  __device__ __forceinline__ float2 apply_c(int m, int y, int z, float2 o) {
    if (xmode == 0) {
      const int x = 2 * m;
      const float g0 = g.at(x, y, z), g1 = g.at(x + 1, y, z);
      const float i0 = cur ? CLARITY_LDG(&cur[w.idx(x, y, z)]) : g0;
      const float i1 = cur ? CLARITY_LDG(&cur[w.idx(x + 1, y, z)]) : g1;
      const float2 r = make_float2(upd(i0, g0, o.x), upd(i1, g1, o.y));
      *reinterpret_cast<float2*>(inext + w.idx(x, y, z)) = r;
      return r;
    }
    const float g0 = g.at(m, y, z);
    const float i0 = cur ? CLARITY_LDG(&cur[w.idx(m, y, z)]) : g0;
    const float r = upd(i0, g0, o.x);
    inext[w.idx(m, y, z)] = r;
    return make_float2(r, 0.f);
  }
    // padding rows / z planes where the result is known to be zero
  __device__ __forceinline__ bool zero_row(int, int) const { return false; }
  __device__ __forceinline__ bool zero_plane(int) const { return false; }
  // rows y0base + BY*j, j < live_rows, can be nonzero (all here)
  __device__ __forceinline__ int live_rows(int, int, int ay) const { return ay; }
  __device__ __forceinline__ void prefetch_row(int y, int z) const {
    if (cur) prefetch_l2_range(cur + w.idx(0, y, z), sizeof(float) * (size_t)w.nx);
    if (y < g.Y && z < g.Z)
      prefetch_l2_range(g.src + ((unsigned)z * g.Y + y) * g.X, sizeof(float) * (size_t)g.X);
  }
  __device__ __forceinline__ void finish() {}
};

// ------------------------------------------------------------ spectral ops
// src/ModulateGPU.cu:63-72 / Convolve.cxx:195-205: out = scale * (a * b),
// no conjugate, a = data, b = OTF; the arithmetic order of
// ComplexMultiplyAndScale (include/internal/Complex.h:95-102) is kept.
// scale2 (optional, device memory) multiplies the 1/N scale: the RL flux
// rescale of the transformed estimate is applied here when the estimate was
// transformed before its scale was known.
struct ModOTF {
  static constexpr bool forward_only = false;
  const float2* CLARITY_RESTRICT H;
  float scale;
  const float* CLARITY_RESTRICT scale2 = nullptr;
  // only the first zn z planes of the input spectrum are nonzero (the rest
  // were never written and are read as zeros)
  int zn = 1 << 30;
  // only the first zout z planes of the output are read by the next pass:
  // the rest are neither inverse-transformed along y0 nor stored
  int zout = 1 << 30;
  // the OTF tile this block will multiply by, into L2 (part p of np)
  __device__ __forceinline__ void prefetch_tile(unsigned base, int tile, int p, int np) const {
    const size_t chunk = ((size_t)tile * 8 / np + 15) & ~size_t(15);
    const size_t off = chunk * p, total = (size_t)tile * 8;
    if (off < total)
      prefetch_l2_range(reinterpret_cast<const char*>(H + base) + off,
                        off + chunk <= total ? chunk : total - off);
  }
  __device__ __forceinline__ float2 apply(long long idx, float2 v) const {
    const float2 h = CLARITY_LDG(&H[idx]);
    const float f = scale2 ? scale * *scale2 : scale;
    return make_float2(f * (v.x * h.x - v.y * h.y), f * (v.x * h.y + v.y * h.x));
  }
  // the same operation with the deferred factor read once (per thread)
  __device__ __forceinline__ ModOTF resolved() const {
    ModOTF r = *this;
    if (scale2) {
      r.scale = scale * CLARITY_LDG(scale2);
      r.scale2 = nullptr;
    }
    return r;
  }
};

// src/WienerDeconvolveGPU.cu:43-49: conj(H) / (|H|^2 + eps), then
// scale * (that * G).
struct ModWiener {
  static constexpr bool forward_only = false;
  const float2* CLARITY_RESTRICT H;
  float eps, scale;
  int zn = 1 << 30;
  int zout = 1 << 30;
  __device__ __forceinline__ void prefetch_tile(unsigned base, int tile, int p, int np) const {
    const size_t chunk = ((size_t)tile * 8 / np + 15) & ~size_t(15);
    const size_t off = chunk * p, total = (size_t)tile * 8;
    if (off < total)
      prefetch_l2_range(reinterpret_cast<const char*>(H + base) + off,
                        off + chunk <= total ? chunk : total - off);
  }
  __device__ __forceinline__ float2 apply(long long idx, float2 v) const {
    const float2 h = CLARITY_LDG(&H[idx]);
    const float mag = h.x * h.x + h.y * h.y;
    const float f = 1.0f / (mag + eps);
    const float a = h.x * f, b = -h.y * f;
    return make_float2(scale * (a * v.x - b * v.y), scale * (a * v.y + b * v.x));
  }
  __device__ __forceinline__ ModWiener resolved() const { return *this; }
};

struct ModForward {
  static constexpr bool forward_only = true;
  int zn = 1 << 30;
  int zout = 1 << 30;
  __device__ __forceinline__ void prefetch_tile(unsigned, int, int, int) const {}
  __device__ __forceinline__ float2 apply(long long, float2 v) const { return v; }
  __device__ __forceinline__ ModForward resolved() const { return *this; }
};

}  // namespace clarity
