// passes_xy_tma.cuh -- the XY inverse (+ epilogue) (+ forward) pass with its
// HBM traffic moved by the Tensor Memory Accelerator.
//
// One block owns the tile (z, y0base .. y0base+TG-1): all AY rows y = y0 +
// BY*j of those TG y0 lines.  At block start one thread issues
//   * one tiled tensor load of the tile's spectrum columns, the box
//     S[k1 = 0..AY)[kg = 0..KG)[z][y0base .. +TG)[ki = 0..W) (33 KB for the
//     512x512x128 box), and
//   * one bulk copy per tile row of the real volume the epilogue reads (the
//     RL estimate or the image),
// both completing on mbarriers, so no thread waits on HBM inside the
// transforms.  The column step then runs one length-AY DFT per thread out of
// shared memory (every column a task of its own: the kx = 0 and kx = M columns
// share one DFT as the real and imaginary parts of one complex column), the
// x passes and the epilogue run as in passes_static.cuh, the epilogue's output
// rows leave by bulk stores, and the forward column step writes the box back
// into the same buffer for one tiled tensor store.
//
// Shared memory per block: the column box, reused in place for the x rows,
// plus the staged real rows (65 KB for 512x512x128, three blocks per SM).
#pragma once
#include "passes_static.cuh"
#ifdef CLARITY_HOST_EMULATION
#include <vector>
#endif

namespace clarity {
namespace st {

template <class SH, int TG>
using TileShape = Shape<typename SH::X, SH::AY, typename SH::Y, typename SH::Z, TG, SH::W>;

template <class SH>
struct XyTma {
  // y0 lines per tile: the box's innermost extent TG*W float2 must be a
  // multiple of 16 bytes
  static constexpr int TG = (SH::W % 2 == 0) ? 1 : 2;
  using T = TileShape<SH, TG>;
  static constexpr int M = SH::M, NX = SH::NX, AY = SH::AY, W = SH::W, KG = SH::KG;
  static constexpr int BOXW = TG * W;  // float2 per (k1, kg) in the box
  static constexpr int BOX_F2 = AY * KG * BOXW;
  static constexpr int ROWS_F2 = TG * T::GSTRIDE;
  static constexpr int BUF_F2_RAW = BOX_F2 > ROWS_F2 ? BOX_F2 : ROWS_F2;
  static constexpr int BUF_F2 = (BUF_F2_RAW + 15) / 16 * 16;  // 128-byte multiple
  static constexpr int NROWS = TG * AY;
  static constexpr int STG_F = NROWS * NX;
  static constexpr int SMEM = BUF_F2 * 8 + STG_F * 4;
  static constexpr int TASKS = TG * M;  // column DFTs per tile
  // x twiddles (M) and the lines' y split twiddles (TG*AY) staged in shared
  // memory when three blocks per SM still fit beside the dynamic tile
  static constexpr int TW_F2 = M + TG * AY;
  static constexpr bool TW_SMEM = 3 * (SMEM + TW_F2 * 8 + 2048 + 1024) <= 228 * 1024;
  static constexpr int THREADS = SH::THREADS;
  static constexpr int BLOCKS = SH::NZ * (SH::BY / TG);
  // usable when the tile fits three 256-thread blocks per SM, every column
  // task has a thread, the rows are whole 16-byte runs and the box is a legal
  // TMA box
  static constexpr bool OK = SMEM <= 72 * 1024 && THREADS == 256 && TASKS <= THREADS &&
                             M % 2 == 0 && M >= 4 &&
                             AY % 2 == 0 &&
                             NX % 4 == 0 && SH::BY % TG == 0 && KG <= 256 && AY <= 256 &&
                             (BOXW * 8) % 16 == 0;
  // box float2 index of column kx of tile line g at k1
  __device__ __forceinline__ static int box(int k1, int kx, int g) {
    return (k1 * KG + kx / W) * BOXW + g * W + kx % W;
  }
};

// Column task c of the tile: line g = c / M; within a line task 0 is the
// packed kx = 0 / kx = M pair, task 1 is kx = M/2 and task 2k (2k+1) is
// kx = k (M - k) for 0 < k < M/2.
__device__ __forceinline__ int task_kx(int cc, int M) {
  const int k = cc >> 1;
  return (cc & 1) ? M - k : k;
}

// Runs a(c, v) for every column task c, then (after a block barrier) b(c, v)
// with the same v: on the GPU v is the task's registers (one task per
// thread); the CPU emulation, one thread per block, keeps every task's v in
// an array.
template <int TASKS, int AY, class A, class B>
__device__ __forceinline__ void per_task_two_phase(const A& a, const B& b) {
#ifndef CLARITY_HOST_EMULATION
  float2 v[AY];
  const int c = threadIdx.x;
  if (c < TASKS) a(c, v);
  __syncthreads();
  if (c < TASKS) b(c, v);
#else
  std::vector<float2> regs((size_t)TASKS * AY);
  for (int c = 0; c < TASKS; ++c) a(c, &regs[(size_t)c * AY]);
  for (int c = 0; c < TASKS; ++c) b(c, &regs[(size_t)c * AY]);
#endif
}

// As per_task_two_phase, and b also gets other(j): row j of the partner
// task c ^ 1 (the column M - kx of the pair), from a warp shuffle on the GPU
// (every task's lane pair shares a warp: TASKS is a multiple of 32 and
// tasks are threads) or from the array in the CPU emulation.  other(j) must
// be called by every thread, in uniform control flow.
template <int TASKS, int AY, class A, class B>
__device__ __forceinline__ void per_task_two_phase_pairs(const A& a, const B& b) {
  static_assert(TASKS % 32 == 0, "a task's pair partner must be in its warp");
#ifndef CLARITY_HOST_EMULATION
  float2 v[AY];
  const int c = threadIdx.x;
  if (c < TASKS) a(c, v);
  __syncthreads();
  auto other = [&](int j) {
    return make_float2(__shfl_xor_sync(0xffffffffu, v[j].x, 1),
                       __shfl_xor_sync(0xffffffffu, v[j].y, 1));
  };
  if (c < TASKS) b(c, v, other);
#else
  std::vector<float2> regs((size_t)TASKS * AY);
  for (int c = 0; c < TASKS; ++c) a(c, &regs[(size_t)c * AY]);
  for (int c = 0; c < TASKS; ++c) {
    const float2* o = &regs[(size_t)(c ^ 1) * AY];
    auto other = [o](int j) { return o[j]; };
    b(c, &regs[(size_t)c * AY], other);
  }
#endif
}

// Inverse column step: box (natural kx) -> x rows (digit-reversed slots),
// with the c2r pair combine of slots k and M - k done as the rows are
// written (the pair's two columns are held by two lanes of one warp).  Only
// rows j < L of each line are written (the later steps read no others).
template <class SH>
__device__ __forceinline__ void cols_inverse_tma(float2* buf, int y0base,
                                                 const float2* __restrict__ twr,
                                                 const float2* twl,
                                                 int L = XyTma<SH>::AY) {
  using X = XyTma<SH>;
  using T = typename X::T;
  constexpr int M = X::M, AY = X::AY, RS = T::ROWSTRIDE;
  auto load = [&](int c, float2* v) {
    const int g = c / M, cc = c - g * M;
    const int y0 = y0base + g;
    const int kx = cc == 0 ? 0 : (cc == 1 ? M / 2 : task_kx(cc, M));
#pragma unroll
    for (int k1 = 0; k1 < AY; ++k1) {
      float2 a = buf[X::box(k1, kx, g)];
      if (k1 != 0 && y0 != 0) a = cmulc(a, twl[g * AY + k1]);
      v[k1] = a;
    }
    if (cc == 0) {
      // A + i B with B the kx = M column: one inverse DFT gives a + i b
#pragma unroll
      for (int k1 = 0; k1 < AY; ++k1) {
        float2 b = buf[X::box(k1, M, g)];
        if (k1 != 0 && y0 != 0) b = cmulc(b, twl[g * AY + k1]);
        v[k1] = make_float2(v[k1].x - b.y, v[k1].y + b.x);
      }
    }
    dft<AY, +1>(v);
  };
  // after the barrier every column is held: the box may be overwritten
  auto store = [&](int c, const float2* v, const auto& other) {
    const int g = c / M, cc = c - g * M;
    float2* rows = buf + g * T::GSTRIDE;
    // pair (k, M - k), 0 < k < M/2: the even task holds X[k], the odd X[M-k]
    const bool pair = cc >= 2, odd = (cc & 1) != 0;
    const int p = cc == 0 ? xp<T>(0)
                          : xp<T>(xrev<T>(cc == 1 ? M / 2 : task_kx(cc, M)));
    const float2 w = pair ? __ldg(&twr[cc >> 1]) : make_float2(1.f, 0.f);
#pragma unroll
    for (int j = 0; j < AY; ++j) {
      if (j >= L) continue;  // L is the same for every thread
      const float2 ov = other(j);
      if (cc == 0) {
        rows[j * RS + p] = make_float2(v[j].x + v[j].y, v[j].x - v[j].y);
      } else if (cc == 1) {
        rows[j * RS + p] = make_float2(2.f * v[j].x, -2.f * v[j].y);
      } else {
        const float2 xa = odd ? ov : v[j];
        const float2 b = conjf2(odd ? v[j] : ov);
        const float2 e = cadd(xa, b);
        const float2 o = cmulc(csub(xa, b), w);
        rows[j * RS + p] = odd ? make_float2(e.x + o.y, -e.y + o.x)
                               : make_float2(e.x - o.y, e.y + o.x);
      }
    }
  };
  per_task_two_phase_pairs<X::TASKS, AY>(load, store);
  __syncthreads();
}

// Forward column step: x rows (digit-reversed slots) -> box (natural kx),
// every kx < KG*W written (slots beyond M are zero).  The r2c split of
// slots k and M - k happens as the columns are read: both tasks of a pair
// read both slots and each keeps its own half.  Rows j >= L of each line
// hold zeros, which the split maps to zeros.
template <class SH>
__device__ __forceinline__ void cols_forward_tma(float2* buf, int y0base,
                                                 const float2* __restrict__ twr,
                                                 const float2* twl,
                                                 int L = XyTma<SH>::AY) {
  using X = XyTma<SH>;
  using T = typename X::T;
  constexpr int M = X::M, AY = X::AY, RS = T::ROWSTRIDE;
  (void)L;
  auto load = [&](int c, float2* v) {
    const int g = c / M, cc = c - g * M;
    const float2* rows = buf + g * T::GSTRIDE;
    if (cc == 0) {
      // kx = 0 and kx = M have real columns a, b: one DFT of a + i b gives
      // P = A + i B with A[k] = (P[k] + conj P[-k]) / 2 and
      // B[k] = (P[k] - conj P[-k]) / 2i, both Hermitian; v keeps their
      // halves: v[k] = A[k] and v[AY-k] = B[k] for 0 < k < AY/2, and the
      // real A, B at k = 0 and AY/2 as the two parts of v[0] and v[AY/2]
      const int p0 = xp<T>(0);
#pragma unroll
      for (int j = 0; j < AY; ++j) {
        const float2 Z0 = rows[j * RS + p0];
        v[j] = make_float2(Z0.x + Z0.y, Z0.x - Z0.y);
      }
      dft<AY, -1>(v);
#pragma unroll
      for (int k = 1; k < AY / 2; ++k) {
        const float2 p = v[k], q = v[AY - k];
        v[k] = make_float2(0.5f * (p.x + q.x), 0.5f * (p.y - q.y));
        v[AY - k] = make_float2(0.5f * (p.y + q.y), 0.5f * (q.x - p.x));
      }
    } else if (cc == 1) {
      const int ph = xp<T>(xrev<T>(M / 2));
#pragma unroll
      for (int j = 0; j < AY; ++j) v[j] = conjf2(rows[j * RS + ph]);
      dft<AY, -1>(v);
    } else {
      // pair (k, M - k): the even task keeps X[k], the odd X[M - k]
      const int k = cc >> 1;
      const bool odd = (cc & 1) != 0;
      const int pa = xp<T>(xrev<T>(k)), pb = xp<T>(xrev<T>(M - k));
      const float2 w = __ldg(&twr[k]);
#pragma unroll
      for (int j = 0; j < AY; ++j) {
        const float2 a = rows[j * RS + pa];
        const float2 b = conjf2(rows[j * RS + pb]);
        const float2 e = make_float2(0.5f * (a.x + b.x), 0.5f * (a.y + b.y));
        const float2 d = csub(a, b);
        const float2 o = make_float2(0.5f * d.y, -0.5f * d.x);
        const float2 wo = cmul(w, o);
        v[j] = odd ? conjf2(csub(e, wo)) : cadd(e, wo);
      }
      dft<AY, -1>(v);
    }
  };
  // after the barrier every row is read: the box may overwrite it
  auto store = [&](int c, const float2* v) {
    const int g = c / M, cc = c - g * M;
    const int y0 = y0base + g;
    const int kx = cc == 0 ? 0 : (cc == 1 ? M / 2 : task_kx(cc, M));
#pragma unroll
    for (int k1 = 0; k1 < AY; ++k1) {
      const float2 w = (k1 == 0 || y0 == 0) ? make_float2(1.f, 0.f) : twl[g * AY + k1];
      if (cc == 0) {
        constexpr int H = AY / 2;
        float2 a, b;
        if (k1 == 0 || k1 == H) {
          a = make_float2(v[k1].x, 0.f);
          b = make_float2(v[k1].y, 0.f);
        } else if (k1 < H) {
          a = v[k1];
          b = v[AY - k1];
        } else {
          a = conjf2(v[AY - k1]);
          b = conjf2(v[k1]);
        }
        buf[X::box(k1, 0, g)] = cmul(a, w);
        buf[X::box(k1, M, g)] = cmul(b, w);
      } else {
        buf[X::box(k1, kx, g)] = cmul(v[k1], w);
      }
    }
  };
  per_task_two_phase<X::TASKS, AY>(load, store);
  // padding slots kx = M+1 .. KG*W-1 of every (k1, g)
  constexpr int PADK = X::KG * X::W - (M + 1);
  if constexpr (PADK > 0) {
    for (int f = threadIdx.x; f < AY * X::TG * PADK; f += CLARITY_BLOCK_STRIDE(SH::THREADS)) {
      const int kx = M + 1 + f % PADK;
      const int rest = f / PADK;
      buf[X::box(rest / X::TG, kx, rest % X::TG)] = make_float2(0.f, 0.f);
    }
  }
}

// Last inverse x pass into the epilogue with the tile row staged in shared
// memory (srow, NX floats); FUSE re-applies forward pass 0.
template <class T, class Epi, bool FUSE, class Skip, bool COMPACT>
__device__ __forceinline__ void x_last_staged(float2* sm, float* stg, Epi& epi, int z, int y0base,
                                              const float2* tw, const Skip& skip,
                                              const int* nf, int L) {
  using X = typename T::X;
  constexpr int R = X::radix(0), span = X::span(0);
  const int total = visit_rows<T, COMPACT>(L) * span;
#pragma unroll 1
  for (int f = threadIdx.x; f < total; f += CLARITY_BLOCK_STRIDE(T::THREADS)) {
    const int rv = f / span;
    const int r = visit_row<T, COMPACT>(rv, L);
    const int i = f - rv * span;
    const int g = r / T::AY, j = r - g * T::AY;
    const int y = y0base + g + T::BY * j;
    float2* row = sm + row_off<T>(r);
    if (skip(r)) {  // known-zero row: its forward transform is zero
      if constexpr (FUSE) {
#pragma unroll
        for (int t = 0; t < R; ++t) row[xp<T>(i + t * span)] = make_float2(0.f, 0.f);
      }
      continue;
    }
    float2 v[R];
#pragma unroll
    for (int t = 0; t < R; ++t) v[t] = row[xp<T>(i + t * span)];
    if (i != 0) {
#pragma unroll
      for (int k = 1; k < R; ++k) v[k] = cmulc(v[k], tw[i * k]);
    }
    dft<R, +1>(v);
    float* srow = stg + r * T::NX;
    const int n = nf[r];
#pragma unroll
    for (int t = 0; t < R; ++t) v[t] = epi.apply_s(i + t * span, y, z, v[t], srow, n);
    if constexpr (FUSE) {
      dft<R, -1>(v);
      if (i != 0) {
#pragma unroll
        for (int k = 1; k < R; ++k) v[k] = cmul(v[k], tw[i * k]);
      }
#pragma unroll
      for (int t = 0; t < R; ++t) row[xp<T>(i + t * span)] = v[t];
    }
  }
}

// The pass kernel.  S box in/out through the tensor map tm (float view of S:
// dims {2*W*BY, NZ, KG, AY}); FUSE = false is the final inverse (no forward
// transform, S is only read).
template <class SH, class Epi, bool FUSE>
__global__ void __launch_bounds__(256, 3)
    ks_xy_tma(Epi epi, CLARITY_GRID_CONST TensorMap tm, const Tables T) {
  CLARITY_PDL_WAIT();  // the previous pass's output is complete and visible
  using X = XyTma<SH>;
  using TS = typename X::T;
  static_assert(X::OK, "shape not supported by the TMA XY pass");
  CLARITY_DYN_SMEM(float2, buf);
  float* stg = reinterpret_cast<float*>(buf + X::BUF_F2);
  __shared__ alignas(8) uint64_t bars[2];
  __shared__ int nf[X::NROWS];
  __shared__ int bulk_ok;
  constexpr int NB = SH::BY / X::TG;
  const int z = blockIdx.x / NB;
  const int y0base = (blockIdx.x - z * NB) * X::TG;
  if (epi.zero_plane(z)) {  // neither read nor written (see Mod::zn)
    if constexpr (requires { epi.finish_skipped(); }) epi.finish_skipped();
    return;
  }
  if (!smem_aligned128(buf)) {    // never expected: refuse rather than fault
    if (threadIdx.x == 0) raise_error(T.err, kErrMisaligned);
    return;
  }
  if (threadIdx.x == 0) {
    int ok = 1;
    for (int r = 0; r < X::NROWS; ++r) {
      const int g = r / X::AY, j = r - g * X::AY;
      const RowRef rr = epi.in_row(y0base + g + SH::BY * j, z);
      nf[r] = rr.nf;
      if (rr.nf > 0 && (((uintptr_t)rr.p & 15u) != 0 || (rr.nf & 3) != 0)) ok = 0;
    }
    bulk_ok = ok;
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    mbar_arrive_expect_tx(&bars[0], (uint32_t)(X::BOX_F2 * 8));
    tma_load_4d(buf, &tm, 2 * SH::W * y0base, z, 0, 0, &bars[0]);
    uint32_t bytes = 0;
    if (bulk_ok)
      for (int r = 0; r < X::NROWS; ++r) bytes += 4u * (uint32_t)nf[r];
    mbar_arrive_expect_tx(&bars[1], bytes);
  }
  __syncwarp();
  if (threadIdx.x < 32 && bulk_ok) {
    for (int r = threadIdx.x; r < X::NROWS; r += CLARITY_ISSUE_LANES) {
      if (nf[r] <= 0) continue;
      const int g = r / X::AY, j = r - g * X::AY;
      const RowRef rr = epi.in_row(y0base + g + SH::BY * j, z);
      bulk_load(stg + r * X::NX, rr.p, 4u * (uint32_t)rr.nf, &bars[1]);
    }
  }
  if (!bulk_ok) {  // rows not 16-byte runs: plain loads
    for (int t = threadIdx.x; t < X::STG_F; t += CLARITY_BLOCK_STRIDE(SH::THREADS)) {
      const int r = t / X::NX, x = t - r * X::NX;
      if (x < nf[r]) {
        const int g = r / X::AY, j = r - g * X::AY;
        stg[t] = __ldg(epi.in_row(y0base + g + SH::BY * j, z).p + x);
      }
    }
  }
  // twiddles into shared memory while the tile is in flight: the lines'
  // y split factors w_ny^(y0*k1) (1 for k1 = 0 or y0 = 0) and, when they fit,
  // the x table w_M^t
  __shared__ float2 s_twl[X::TG * X::AY];
  __shared__ float2 s_twx[X::TW_SMEM ? X::M : 1];
  for (int t = threadIdx.x; t < X::TG * X::AY; t += CLARITY_BLOCK_STRIDE(SH::THREADS)) {
    const int g = t / X::AY, k1 = t - g * X::AY, y0 = y0base + g;
    s_twl[t] = (k1 != 0 && y0 != 0) ? __ldg(&T.twny[y0 * k1]) : make_float2(1.f, 0.f);
  }
  if constexpr (X::TW_SMEM)
    for (int t = threadIdx.x; t < X::M; t += CLARITY_BLOCK_STRIDE(SH::THREADS)) s_twx[t] = __ldg(&T.twx[t]);
  const float2* twx = X::TW_SMEM ? s_twx : T.twx;
  __syncthreads();
  bool ok = mbar_wait(&bars[0], 0, T.err);
  if (!ok) {
    mbar_wait(&bars[0], 0, nullptr);  // give copies in flight a last chance
    mbar_wait(&bars[1], 0, nullptr);
    return;
  }
  // rows j >= L of every line are outside the image (zero for this epilogue)
  int L = SH::AY;
  if constexpr (Epi::has_zero_rows) L = epi.live_rows(y0base, SH::BY, SH::AY);
  constexpr bool CP = Epi::has_zero_rows;
  cols_inverse_tma<SH>(buf, y0base, T.twr, s_twl, L);
  const RowSkip<TS, Epi> skip{epi, z, y0base};
  x_inverse_down_to<TS, 1, RowSkip<TS, Epi>, CP>(buf, twx, skip, L);
  if (!mbar_wait(&bars[1], 0, T.err)) {
    mbar_wait(&bars[1], 0, nullptr);
    return;
  }
  x_last_staged<TS, Epi, FUSE, RowSkip<TS, Epi>, CP>(buf, stg, epi, z, y0base, twx, skip,
                                                     nf, L);
  if constexpr (Epi::kStoreRows) {
    // the epilogue's output rows, written in place of its input, leave by
    // bulk stores while the forward transform runs
    fence_smem_to_async();
    __syncthreads();
    if (threadIdx.x < 32) {
      for (int r = threadIdx.x; r < X::NROWS; r += CLARITY_ISSUE_LANES) {
        const int g = r / X::AY, j = r - g * X::AY;
        float* dst = epi.out_row(y0base + g + SH::BY * j, z);
        if (((uintptr_t)dst & 15u) == 0) {
          bulk_store(dst, stg + r * X::NX, 4u * X::NX);
        } else {
          for (int x = 0; x < X::NX; ++x) dst[x] = stg[r * X::NX + x];
        }
      }
      bulk_commit();
    }
  }
  if constexpr (FUSE) {
    if constexpr (CP) {
      // rows j >= L of each group are zero
      const int dead = X::TG * (SH::AY - L) * TS::ROWSTRIDE;
      for (int t = threadIdx.x; t < dead; t += CLARITY_BLOCK_STRIDE(SH::THREADS)) {
        const int rd = t / TS::ROWSTRIDE, e = t - rd * TS::ROWSTRIDE;
        const int g = rd / (SH::AY - L), j = L + (rd - g * (SH::AY - L));
        buf[g * TS::GSTRIDE + j * TS::ROWSTRIDE + e] = make_float2(0.f, 0.f);
      }
    }
    __syncthreads();
    x_forward_from<TS, 1, RowSkip<TS, Epi>, CP>(buf, twx, skip, L);
    cols_forward_tma<SH>(buf, y0base, T.twr, s_twl, L);
    fence_smem_to_async();
    __syncthreads();
    if (threadIdx.x == 0) {
      tma_store_4d(&tm, 2 * SH::W * y0base, z, 0, 0, buf);
      bulk_commit();
    }
  }
  if (threadIdx.x < 32) bulk_wait_read_all();  // shared sources read before exit
  epi.finish();
}

}  // namespace st
}  // namespace clarity
