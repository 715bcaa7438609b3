// static_dispatch.cuh -- compile-time specialised shapes and the launch
// helpers that use them when a plan matches (else the generic kernels run).
//
// Shapes (work box x*y*z -> x radices, Ay, y0 radices, z radices, G, W),
// exactly the plans the planner produces for these boxes:
//   512x512x128   (256x256x64 image + same-size PSF): 16.16, 16, 8.4, 16.8, 2, 2
//   128x128x64    (64x64x32 image + same-size PSF):   8.8,   16, 8,   8.8,  1, 4
//   1024x1024x256 (512x512x128 image + PSF):          8.8.8, 16, 8.8, 16.16, 2, 1
//   64x64x32      (small test box):                  8.4,   16, 4,   8.4,  4, 1
#pragma once
#include "engine.hpp"
#include "ops.cuh"
#include "passes_static.cuh"
#include "passes_xy_tma.cuh"

namespace clarity {

using ShapeW512 = st::Shape<st::Rad<16, 16>, 16, st::Rad<8, 4>, st::Rad<16, 8>, 2, 2>;
using ShapeW128 = st::Shape<st::Rad<8, 8>, 16, st::Rad<8>, st::Rad<8, 8>, 1, 4>;
// The 1024x1024x256 box's XY and z tiles (133 and 128 KB) leave room for one
// block per SM, so its XY blocks run CLARITY_W1024_THREADS threads and its
// FP32 z blocks CLARITY_W1024_Z_THREADS (both measured against 256; more XY
// threads spill registers).  The tensor-core z form keeps the XY count.
#ifndef CLARITY_W1024_THREADS
#define CLARITY_W1024_THREADS 512
#endif
#ifndef CLARITY_W1024_Z_THREADS
#define CLARITY_W1024_Z_THREADS 1024
#endif
using ShapeW1024 = st::Shape<st::Rad<8, 8, 8>, 16, st::Rad<8, 8>, st::Rad<16, 16>, 2, 1,
                             CLARITY_W1024_THREADS, CLARITY_W1024_Z_THREADS>;
using ShapeW64 = st::Shape<st::Rad<8, 4>, 16, st::Rad<4>, st::Rad<8, 4>, 4, 1>;

// The 512x512x128 box keeps its TMA XY pass with shared-memory twiddles and
// three blocks per SM; a tile change that breaks this fails to compile.
static_assert(st::XyTma<ShapeW512>::OK && st::XyTma<ShapeW512>::TW_SMEM,
              "the 512x512x128 XY tile no longer fits three TMA blocks per SM");

template <class... SHs>
struct ShapeList {};
using StaticShapes = ShapeList<ShapeW512, ShapeW128, ShapeW1024, ShapeW64>;

inline st::Tables tables_of(const PlanEntry& pe) {
  const VolPlan& P = pe.P;
  return st::Tables{pe.tw + P.ax.tw_off, pe.tw + P.ayB.tw_off, pe.tw + P.az.tw_off,
                    pe.tw + P.tw_r2c_off, pe.tw + P.tw_ny_off, pe.err};
}

template <class K>
inline cudaError_t allow_smem_st(K kernel, int smem) {
  return smem_opt_in(reinterpret_cast<const void*>(kernel), smem);
}

// The TMA XY pass (passes_xy_tma.cuh) serves epilogues with a staged form
// unless CLARITY_XY_TMA=0.
bool xy_tma_enabled();
template <class F>
constexpr bool xy_staged() {
  if constexpr (requires { F::kStaged; }) return F::kStaged;
  else return false;
}

// Tensor map of the spectrum S as floats {2*W*BY, NZ, KG, AY} with the box of
// one XY tile.
template <class SH>
inline bool encode_s_map(TensorMap* tm, const float2* S) {
  using X = st::XyTma<SH>;
  const unsigned long long row = 2ull * SH::W * SH::BY;
  const unsigned long long dim[4] = {row, (unsigned long long)SH::NZ,
                                     (unsigned long long)SH::KG, (unsigned long long)SH::AY};
  const unsigned long long stride[3] = {row * 4, row * 4 * SH::NZ,
                                        row * 4 * SH::NZ * SH::KG};
  const unsigned box[4] = {2u * X::BOXW, 1u, (unsigned)SH::KG, (unsigned)SH::AY};
  return encode_tensor_f32_4d(tm, S, dim, stride, box);
}

// Launches the TMA XY pass when shape, epilogue and buffers allow it.
template <class SH, bool FUSE, class F>
inline bool try_xy_tma(const PlanEntry& pe, cudaStream_t st, const F& fn, const float2* S,
                       int family, cudaError_t* err) {
  using X = st::XyTma<SH>;
  if constexpr (X::OK && xy_staged<F>()) {
    if (!xy_tma_enabled()) return false;
    // the map depends only on S: encoded once per buffer
    static thread_local const float2* map_s = nullptr;
    static thread_local TensorMap tm;
    if (S != map_s) {
      if (!encode_s_map<SH>(&tm, S)) {
        map_s = nullptr;
        return false;
      }
      map_s = S;
    }
    auto k = st::ks_xy_tma<SH, F, FUSE>;
    *err = allow_smem_st(k, X::SMEM);
    if (*err != cudaSuccess) return true;
    const st::Tables T = tables_of(pe);
    // planes known to be zero need no block at all
    int nz = SH::NZ;
    if constexpr (requires { fn.live_planes(1); }) nz = fn.live_planes(SH::NZ);
    const int blocks = nz * (SH::BY / X::TG);
    if (blocks <= 0) return true;
    note_launch_begin(family, st);
    CLARITY_LAUNCH_PDL(k, blocks, SH::THREADS, X::SMEM, st, pdl_enabled())(fn, tm, T);
    note_launch_end(family, st);
    *err = cudaGetLastError();
    return true;
  } else {
    (void)pe; (void)st; (void)fn; (void)S; (void)family; (void)err;
    return false;
  }
}

// Kernel families that may use the specialised kernels: bit KIND of the
// CLARITY_STATIC environment variable (default: all).  Clearing bits selects
// the runtime-generic kernels, which tests use to cover both paths.
int static_family_mask();

// kind: 0 xy forward, 1 z, 2 xy inverse+forward, 3 xy inverse
template <class SH, int KIND, class F>
inline bool try_static(const PlanEntry& pe, cudaStream_t st, const F& fn, float2* Sa,
                       const float2* Sb, cudaError_t* err) {
  if (!(static_family_mask() & (1 << KIND))) return false;
  if (!st::matches<SH>(pe.P)) return false;
  const st::Tables T = tables_of(pe);
  if constexpr (KIND == 0) {
    auto k = st::ks_xy_forward<SH, F>;
    *err = allow_smem_st(k, SH::XY_SMEM);
    if (*err != cudaSuccess) return true;
    note_launch_begin(KK_XY_FORWARD, st);
    CLARITY_LAUNCH(k, pe.P.xy_blocks, SH::THREADS, SH::XY_SMEM, st)(fn, Sa, T);
    note_launch_end(KK_XY_FORWARD, st);
  } else if constexpr (KIND == 1) {
    if constexpr (SH::Y_PER_LINE) {
      auto k = st::ks_z2<SH, F>;
      *err = allow_smem_st(k, SH::Z2_SMEM);
      if (*err != cudaSuccess) return true;
      note_launch_begin(KK_Z, st);
      CLARITY_LAUNCH_PDL(k, pe.P.z_blocks, SH::THREADS, SH::Z2_SMEM, st, pdl_enabled())(fn, Sb,
                                                                                     Sa, T);
      note_launch_end(KK_Z, st);
    } else {
      auto k = st::ks_z<st::ZThreads<SH>, F>;
      int threads = SH::Z_THREADS;
      if constexpr (st::kTcZ<SH> && !F::forward_only) {
        // the precision form: tensor-core first z stage (the OTF stays FP32)
        const int prec = dft_precision();
        if (prec == st::kDftF16Split) k = st::ks_z<SH, F, st::kDftF16Split>;
        if (prec == st::kDftBF16Split) k = st::ks_z<SH, F, st::kDftBF16Split>;
        if (prec != st::kDftF32) threads = SH::THREADS;
      }
      *err = allow_smem_st(k, SH::Z_SMEM);
      if (*err != cudaSuccess) return true;
      note_launch_begin(KK_Z, st);
      CLARITY_LAUNCH(k, pe.P.z_blocks, threads, SH::Z_SMEM, st)(fn, Sb, Sa, T);
      note_launch_end(KK_Z, st);
    }
  } else if constexpr (KIND == 2) {
    if (try_xy_tma<SH, true>(pe, st, fn, Sa, family_of<F, KK_XY_INV_FWD>(), err)) return true;
    auto k = st::ks_xy_inv_fwd<SH, F>;
    *err = allow_smem_st(k, SH::XY_SMEM);
    if (*err != cudaSuccess) return true;
    note_launch_begin(family_of<F, KK_XY_INV_FWD>(), st);
    CLARITY_LAUNCH(k, pe.P.xy_blocks, SH::THREADS, SH::XY_SMEM, st)(fn, Sa, T);
    note_launch_end(family_of<F, KK_XY_INV_FWD>(), st);
  } else {
    if (try_xy_tma<SH, false>(pe, st, fn, Sb, KK_XY_INVERSE, err)) return true;
    auto k = st::ks_xy_inverse<SH, F>;
    *err = allow_smem_st(k, SH::XY_SMEM);
    if (*err != cudaSuccess) return true;
    note_launch_begin(KK_XY_INVERSE, st);
    CLARITY_LAUNCH(k, pe.P.xy_blocks, SH::THREADS, SH::XY_SMEM, st)(fn, Sb, T);
    note_launch_end(KK_XY_INVERSE, st);
  }
  *err = cudaGetLastError();
  return true;
}

template <int KIND, class F, class... SHs>
inline bool try_static_all(ShapeList<SHs...>, const PlanEntry& pe, cudaStream_t st,
                           const F& fn, float2* Sa, const float2* Sb, cudaError_t* err) {
  return (try_static<SHs, KIND>(pe, st, fn, Sa, Sb, err) || ...);
}

// Entry points used by launch.cuh; each returns true when a specialised
// kernel was launched (the error, if any, in *err).
template <class F>
bool static_xy_forward(const PlanEntry& pe, cudaStream_t st, const F& f, float2* S,
                       cudaError_t* err) {
  return try_static_all<0>(StaticShapes{}, pe, st, f, S, nullptr, err);
}
template <class F>
bool static_z(const PlanEntry& pe, cudaStream_t st, const F& f, const float2* Sin,
              float2* Sout, cudaError_t* err) {
  return try_static_all<1>(StaticShapes{}, pe, st, f, Sout, Sin, err);
}
template <class F>
bool static_xy_inv_fwd(const PlanEntry& pe, cudaStream_t st, const F& f, float2* S,
                       cudaError_t* err) {
  return try_static_all<2>(StaticShapes{}, pe, st, f, S, nullptr, err);
}
template <class F>
bool static_xy_inverse(const PlanEntry& pe, cudaStream_t st, const F& f, const float2* S,
                       cudaError_t* err) {
  return try_static_all<3>(StaticShapes{}, pe, st, f, nullptr, S, err);
}

}  // namespace clarity
