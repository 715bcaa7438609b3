// nn.cu -- kernels of the learned-start network: a 3-D U-Net on channels-last
// BF16 activations with FP32 accumulation.
//
// * conv3: 3x3x3 convolution (zero padding 1) as an implicit GEMM on the
//   tensor cores (mma.sync m16n8k16 bf16 -> f32).  M = voxels (128 per block),
//   N = output channels, K = 27 taps x input channels.  The input may be the
//   concatenation of a full-resolution tensor and a half-resolution tensor read
//   through nearest upsampling (the decoder's skip + up path), so neither the
//   upsampled nor the concatenated tensor is ever stored.  A- and B-tiles move
//   global -> shared by cp.async (zero-fill at the volume border) in a two-stage
//   pipeline, fragments by ldmatrix.  Epilogue: bias, ReLU, or a ReLU-derivative
//   mask (backward data), BF16 store.  The backward data pass is the same
//   kernel with the mirrored, transposed weights.
// * conv3_wgrad: dW[co][tap][ci] = sum_v dy[v][co] in(v + tap)[ci], the same
//   implicit-GEMM tiles with K = voxels, split over blocks and summed with FP32
//   atomics.
// * SIMT kernels: the 1 -> 16 input convolution, the 16 -> 1 head with the loss,
//   pooling, the gradient merges, bias sums, Adam, weight packing.
//
// Layout: activation [v][c], v = (z*H + y)*W + x; weights [co][tap][ci] with
// tap = (dz+1)*9 + (dy+1)*3 + (dx+1).  Channel counts of the tensor-core
// kernels are multiples of 16.
#include <cuda_bf16.h>

#include <cstdint>
#include <cstdlib>
#include <cstring>

#include "engine.hpp"
#include "launch_macro.cuh"
#include "ops.cuh"

namespace clarity {
namespace nn {

using bf16 = __nv_bfloat16;

struct Conv3Args {
  const bf16* x1;  // full-resolution input [v][c1]
  int c1;
  const bf16* x2;  // optional half-resolution input [u][c2] (nearest upsampled), or nullptr
  int c2;
  int D, H, W;     // output (= full-resolution input) dims
  int D2, H2, W2;  // x2 dims
  const bf16* w;   // [cout][27][c1 + c2]
  const float* bias;
  int cout;
  int relu;
  const bf16* mask;  // optional [v][cout]: result *= (mask > 0)
  bf16* y;           // [v][cout]
  int* err = nullptr;  // error word for bounded waits that give up (tcgen05 path)
};

constexpr int kBM = 128;   // voxels per block
constexpr int kRow = 24;   // smem row pitch in bf16 (48 B: conflict-free ldmatrix)

__device__ __forceinline__ void tap_offset(int t, int* dz, int* dy, int* dx) {
  *dz = t / 9 - 1;
  *dy = (t / 3) % 3 - 1;
  *dx = t % 3 - 1;
}

// Source of 8 consecutive input channels [c, c+8) at shifted voxel
// (z, y, x); nullptr outside the volume (zero padding).
__device__ __forceinline__ const bf16* in_chunk(const Conv3Args& a, int z, int y, int x, int c) {
  if (z < 0 || y < 0 || x < 0 || z >= a.D || y >= a.H || x >= a.W) return nullptr;
  if (c < a.c1) return a.x1 + ((size_t)((z * a.H + y) * a.W + x) * a.c1 + c);
  const int zz = z >> 1, yy = y >> 1, xx = x >> 1;
  return a.x2 + ((size_t)((zz * a.H2 + yy) * a.W2 + xx) * a.c2 + (c - a.c1));
}

#ifndef CLARITY_HOST_EMULATION
__device__ __forceinline__ uint32_t su32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
// 16-byte global -> shared copy; src nullptr -> zero fill
__device__ __forceinline__ void cp16(void* dst, const void* src, const void* any_valid) {
  const int n = src ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(su32(dst)),
               "l"(src ? src : any_valid), "r"(n)
               : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}
__device__ __forceinline__ void ldm_x4(uint32_t* r, const void* p) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(su32(p)));
}
__device__ __forceinline__ void ldm_x4_t(uint32_t* r, const void* p) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(su32(p)));
}
__device__ __forceinline__ void mma16816(float* c, const uint32_t* a, const uint32_t* b) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, "
      "{%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}
#else
inline void cp16(void* dst, const void* src, const void*) {
  if (src) std::memcpy(dst, src, 16);
  else std::memset(dst, 0, 16);
}
inline void cp_commit() {}
template <int N>
inline void cp_wait() {}
#endif

// out[v][co] = sum_{tap, c} in(v + tap)[c] w[co][tap][c] (+ bias, ReLU / mask).
// One block computes a 2x8x8 (z, y, x) tile of output voxels for BN output
// channels.  Per 16-channel input chunk it stages the tile's 4x10x10 halo
// and all 27 taps' weights in shared memory once; the 27 tap GEMMs then read
// their A rows from the halo at shifted positions (each lane of ldmatrix
// supplies its own row address), so an input voxel is read from HBM/L2 once
// per chunk instead of once per tap.  128 threads; warp w owns tile voxels
// [32w, 32w + 32) (tile z = w / 2, y rows 4(w % 2) .. +3).
constexpr int kTZ = 2, kTY = 8, kTX = 8;
constexpr int kHZ = kTZ + 2, kHY = kTY + 2, kHX = kTX + 2;
constexpr int kHalo = kHZ * kHY * kHX;  // 400 voxels

template <int BN>
struct Conv3Smem {
  static constexpr int HALO = kHalo * kRow;     // bf16 elements
  static constexpr int WTS = 27 * BN * kRow;
  static constexpr int BYTES = (HALO + WTS) * 2;
};

template <int BN>
__global__ void __launch_bounds__(128) k_conv3(const Conv3Args a) {
  static_assert(BN % 16 == 0 && BN <= 64, "BN: 16, 32, 48 or 64");
  CLARITY_DYN_SMEM(bf16, sm);
  bf16* Hs = sm;                              // [halo voxel][24]
  bf16* Ws = sm + Conv3Smem<BN>::HALO;        // [tap][n][24]
  const int cin = a.c1 + a.c2;
  const int nchunks = cin / 16;
  const int ntx = (a.W + kTX - 1) / kTX, nty = (a.H + kTY - 1) / kTY;
  const int tile = blockIdx.x;
  const int tx0 = (tile % ntx) * kTX;
  const int ty0 = ((tile / ntx) % nty) * kTY;
  const int tz0 = (tile / (ntx * nty)) * kTZ;
  const int co0 = blockIdx.y * BN;

  auto load = [&](int cc) {
    for (int q = threadIdx.x; q < 2 * kHalo; q += CLARITY_BLOCK_STRIDE(128)) {
      const int h = q >> 1, half = q & 1;
      const int hx = h % kHX, hy = (h / kHX) % kHY, hz = h / (kHX * kHY);
      const bf16* src = in_chunk(a, tz0 - 1 + hz, ty0 - 1 + hy, tx0 - 1 + hx, cc * 16 + half * 8);
      cp16(&Hs[h * kRow + half * 8], src, a.x1);
    }
    for (int q = threadIdx.x; q < 27 * BN * 2; q += CLARITY_BLOCK_STRIDE(128)) {
      const int half = q & 1, tn = q >> 1;
      const int n = tn % BN, t = tn / BN;
      const bf16* src = a.w + ((size_t)(co0 + n) * 27 + t) * cin + cc * 16 + half * 8;
      cp16(&Ws[(t * BN + n) * kRow + half * 8], src, a.x1);
    }
    cp_commit();
  };

#ifndef CLARITY_HOST_EMULATION
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // halo index of this lane's A row for m tile i, at tap offset 0
  int hrow[2];
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    const int m = warp * 32 + i * 16 + (lane & 15);
    const int tx = m % kTX, ty = (m / kTX) % kTY, tz = m / (kTX * kTY);
    hrow[i] = ((tz + 1) * kHY + (ty + 1)) * kHX + (tx + 1);
  }
  float acc[2][BN / 8][4];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < BN / 8; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.f;
  for (int cc = 0; cc < nchunks; ++cc) {
    load(cc);
    cp_wait<0>();
    __syncthreads();
#pragma unroll 1
    for (int t = 0; t < 27; ++t) {
      const int toff = ((t / 9 - 1) * kHY + ((t / 3) % 3 - 1)) * kHX + (t % 3 - 1);
      uint32_t af[2][4];
#pragma unroll
      for (int i = 0; i < 2; ++i)
        ldm_x4(af[i], &Hs[(hrow[i] + toff) * kRow + (lane >> 4) * 8]);
      const bf16* wt = Ws + t * BN * kRow;
#pragma unroll
      for (int j = 0; j < BN / 8; j += 2) {
        uint32_t bfr[4];
        ldm_x4(bfr, &wt[(j * 8 + (lane & 7) + (lane >> 4) * 8) * kRow + ((lane >> 3) & 1) * 8]);
#pragma unroll
        for (int i = 0; i < 2; ++i) {
          mma16816(acc[i][j], af[i], bfr);
          mma16816(acc[i][j + 1], af[i], bfr + 2);
        }
      }
    }
    __syncthreads();
  }
  // epilogue: acc[i][j] holds tile rows g, g+8 (g = lane/4) and channels 2(lane%4), +1
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int m = warp * 32 + i * 16 + (lane >> 2) + h * 8;
      const int x = tx0 + m % kTX, y = ty0 + (m / kTX) % kTY, z = tz0 + m / (kTX * kTY);
      if (x >= a.W || y >= a.H || z >= a.D) continue;
      const long long v = ((long long)z * a.H + y) * a.W + x;
#pragma unroll
      for (int j = 0; j < BN / 8; ++j) {
        const int co = co0 + j * 8 + (lane & 3) * 2;
        float r0 = acc[i][j][2 * h], r1 = acc[i][j][2 * h + 1];
        if (a.bias) {
          r0 += a.bias[co];
          r1 += a.bias[co + 1];
        }
        if (a.relu) {
          r0 = fmaxf(r0, 0.f);
          r1 = fmaxf(r1, 0.f);
        }
        const size_t o = (size_t)v * a.cout + co;
        if (a.mask) {
          const __nv_bfloat162 mk = *reinterpret_cast<const __nv_bfloat162*>(a.mask + o);
          if (!(__bfloat162float(mk.x) > 0.f)) r0 = 0.f;
          if (!(__bfloat162float(mk.y) > 0.f)) r1 = 0.f;
        }
        *reinterpret_cast<__nv_bfloat162*>(a.y + o) = __floats2bfloat162_rn(r0, r1);
      }
    }
#else
  // host emulation: the same tiles, multiplied with scalar loops
  static thread_local float accs[kTZ * kTY * kTX][64];
  for (int r = 0; r < 128; ++r)
    for (int n = 0; n < BN; ++n) accs[r][n] = 0.f;
  for (int cc = 0; cc < nchunks; ++cc) {
    load(cc);
    for (int t = 0; t < 27; ++t) {
      const int toff = ((t / 9 - 1) * kHY + ((t / 3) % 3 - 1)) * kHX + (t % 3 - 1);
      for (int m = 0; m < 128; ++m) {
        const int tx = m % kTX, ty = (m / kTX) % kTY, tz = m / (kTX * kTY);
        const int hr = ((tz + 1) * kHY + (ty + 1)) * kHX + (tx + 1) + toff;
        for (int n = 0; n < BN; ++n) {
          float acc1 = 0.f;
          for (int k = 0; k < 16; ++k)
            acc1 += __bfloat162float(Hs[hr * kRow + k]) *
                    __bfloat162float(Ws[(t * BN + n) * kRow + k]);
          accs[m][n] += acc1;
        }
      }
    }
  }
  for (int m = 0; m < 128; ++m) {
    const int x = tx0 + m % kTX, y = ty0 + (m / kTX) % kTY, z = tz0 + m / (kTX * kTY);
    if (x >= a.W || y >= a.H || z >= a.D) continue;
    const long long v = ((long long)z * a.H + y) * a.W + x;
    for (int n = 0; n < BN; ++n) {
      const int co = co0 + n;
      float xv = accs[m][n];
      if (a.bias) xv += a.bias[co];
      if (a.relu) xv = fmaxf(xv, 0.f);
      const size_t o = (size_t)v * a.cout + co;
      if (a.mask && !(__bfloat162float(a.mask[o]) > 0.f)) xv = 0.f;
      a.y[o] = __float2bfloat16_rn(xv);
    }
  }
#endif
}

// ------------------------------------------------- tcgen05 convolution
// The same convolution on the 5th-generation tensor cores, for volumes whose
// width is a multiple of 32.  One MMA computes 128 output voxels -- a tile of
// tx consecutive x voxels by ty = 128 / tx rows (tx = 128, 64 or 32) -- for BN
// output channels, accumulating in tensor memory (TMEM).  A work item is R
// such tiles stacked along y in one z plane; a persistent block takes items
// round-robin.  For each item the reduction runs over units (16-channel
// chunk, dz): per unit
//   * the load warp brings, by TMA, the unit's input slab (the plane z + dz - 1,
//     rows y0 - 1 .. y0 + R ty, columns x0 - 1 .. x0 + tx, 16 channels; zero
//     outside the volume; for a chunk of the half-resolution input the
//     matching coarse slab) and the 9 taps' weights of that dz into a stage;
//   * eight window warps (two per TMEM lane quarter) turn the slab into the A
//     operands in TMEM: thread m (TMEM lane m = MMA row m) reads its voxel's 16
//     channels from the slab and its x neighbours arrive by warp shuffles, so
//     every tap's shifted window (3 x shifts by S start rows) is written once
//     with tcgen05.st;
//   * one issuing thread per MMA tile (R of them) issues that tile's 9 MMAs
//     (A from TMEM, B = the taps' weights from shared memory) and commits them
//     to the barriers that free the stage and the window buffer.  A single
//     thread issues one tcgen05.mma about every 46 cycles whatever N is, so
//     with N = 16 only several issuers keep the tensor cores busy;
//   * four epilogue warps read a finished item's accumulators (tcgen05.ld),
//     add bias, apply ReLU or the mask and store BF16, while the MMAs of the
//     next item run into the other accumulator buffer.
// Shared memory holds kTmStages stages; TMEM holds two window buffers and one
// or two accumulator buffers.  Every wait is bounded: a wait that runs out
// records a timeout in the error word and sets the block's abort flag, the
// other roles stop at their next wait, in-flight copies and MMAs are waited
// for (again bounded) and the TMEM is freed.
#ifndef CLARITY_HOST_EMULATION
// warps 0-3 epilogue, 4-11 windows (two per TMEM lane quarter), 12 loads,
// 13-16 MMA issue (one per MMA tile of an item)
constexpr int kTmWinWarps = 8;
constexpr int kTmLoadWarp = 4 + kTmWinWarps;
constexpr int kTmIssueWarp = kTmLoadWarp + 1;
constexpr int kTmIssuers = 4;
constexpr int kTmThreads = 32 * (kTmIssueWarp + kTmIssuers);
constexpr int kTmStages = 4;
constexpr int kTmCols = 512;     // TMEM columns the block allocates
constexpr long long kTmWaitLimit = 1ll << 22;  // polls of an mbarrier before giving up
constexpr unsigned kFull = 0xffffffffu;

struct TmGeom {
  int tx, ty, R, rows, S;    // MMA tile tx x ty voxels; R tiles per item; S window rows
  int nxb, nyb, nnb, items;  // items: x blocks x y blocks x z x channel blocks
  int na;                    // accumulator buffers (1 or 2)
  int cw1, cw2;              // slab row lengths (voxels) of the full- and half-resolution inputs
  uint32_t stage, wofs;      // bytes of a stage; offset of its weights
  uint32_t tx1, tx2;         // bytes a stage receives for a full- / half-resolution chunk
  uint32_t acc_cols, win_cols;
};

// Shared-memory matrix descriptor: K-major, no swizzle, 16-byte rows with
// 8-row core matrices 128 bytes apart (SBO) and the second 8 K-elements
// lbo bytes away (LBO); version 1 (bits 46-47) as sm_100 requires.
__device__ __forceinline__ uint64_t tc_sdesc(uint32_t saddr, uint32_t lbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)(128u >> 4) << 32) | ((uint64_t)1 << 46);
}
// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both
// K-major, N >> 3 at bit 17, M >> 4 at bit 24.
constexpr uint32_t tc_idesc(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) |
         ((uint32_t)(M >> 4) << 24);
}
// D (TMEM) (+)= A (TMEM, 128 lanes x 16 BF16) x B (shared memory descriptor)
__device__ __forceinline__ void tc_mma_ts(uint32_t d, uint32_t a, uint64_t b, uint32_t id,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
      ::"r"(d), "r"(a), "l"(b), "r"(id), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
}
__device__ __forceinline__ void tc_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
               ::"r"(su32(bar)) : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_ld16(uint32_t taddr, uint32_t* v) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
      "%11, %12, %13, %14, %15}, [%16];\n"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
        "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
        "=r"(v[14]), "=r"(v[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tc_st8(uint32_t taddr, const uint32_t* v) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};"
      ::"r"(taddr), "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]),
        "r"(v[7])
      : "memory");
}
__device__ __forceinline__ void tc_wait_st() {
  asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tm_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(su32(bar)) : "memory");
}
// Bounded wait that also gives up when another role of the block has
// aborted; the role that runs out of polls records the timeout.
__device__ __forceinline__ bool tm_wait(uint64_t* bar, uint32_t parity, volatile int* abort,
                                        int* err) {
  for (long long it = 0; it < kTmWaitLimit; ++it) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((it & 255) == 255 && *abort) return false;
  }
  *abort = 1;
  raise_error(err, kErrWaitTimeout);
  return false;
}

// Item -> (z, y0, x0, first output channel)
struct TmItem {
  int z, y0, x0, co0;
};
__device__ __forceinline__ TmItem tm_item(const TmGeom& g, int item, int bn) {
  int r = item;
  const int nb = r % g.nnb;
  r /= g.nnb;
  const int xb = r % g.nxb;
  r /= g.nxb;
  const int yb = r % g.nyb;
  return TmItem{r / g.nyb, yb * g.rows, xb * g.tx, nb * bn};
}

// 16 channels of the slab voxel (hr, hc) (halo coordinates: row 0 = y0 - 1,
// column 0 = x0 - 1), from the stage's 32-byte-swizzled slab.  For a
// half-resolution chunk the voxel's coarse parent is read.
__device__ __forceinline__ void tm_slab(const unsigned char* st, const TmGeom& g, bool full,
                                        int y0, int x0, int hr, int hc, uint32_t* v) {
  int off;
  if (full) {
    off = (hr * g.cw1 + hc) * 32;
  } else {
    const int yr = ((y0 - 1 + hr) >> 1) - ((y0 - 1) >> 1);
    const int xc = ((x0 - 1 + hc) >> 1) - ((x0 - 1) >> 1);
    off = (yr * g.cw2 + xc) * 32;
  }
  const int sw = (off >> 7) & 1;  // the swizzle exchanges the halves when bit 7 is set
  const uint4 lo = *reinterpret_cast<const uint4*>(st + off + 16 * sw);
  const uint4 hi = *reinterpret_cast<const uint4*>(st + off + 16 * (sw ^ 1));
  v[0] = lo.x; v[1] = lo.y; v[2] = lo.z; v[3] = lo.w;
  v[4] = hi.x; v[5] = hi.y; v[6] = hi.z; v[7] = hi.w;
}

template <int BN>
__global__ void __launch_bounds__(kTmThreads, 1)
    k_conv3_tm(const Conv3Args a, const TmGeom g, CLARITY_GRID_CONST TensorMap m1,
               CLARITY_GRID_CONST TensorMap m2, CLARITY_GRID_CONST TensorMap mw) {
  static_assert(BN % 16 == 0 && BN >= 16 && BN <= 128, "BN: a multiple of 16 up to 128");
  extern __shared__ unsigned char tm_raw[];
  unsigned char* base = tm_raw + ((1024u - (su32(tm_raw) & 1023u)) & 1023u);
  uint64_t* full = reinterpret_cast<uint64_t*>(base + kTmStages * g.stage);
  uint64_t* empty = full + kTmStages;
  uint64_t* wfull = empty + kTmStages;  // [2] window buffer written
  uint64_t* wempty = wfull + 2;         // [2] window buffer read by its MMAs
  uint64_t* afull = wempty + 2;         // [2] accumulators complete
  uint64_t* aempty = afull + 2;         // [2] accumulators read out
  uint64_t* drain = aempty + 2;         // [kTmIssuers]
  uint32_t* tslot = reinterpret_cast<uint32_t*>(drain + kTmIssuers);
  volatile int* abort = reinterpret_cast<volatile int*>(tslot + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nunits = 3 * ((a.c1 + a.c2) / 16);
  if (warp == kTmLoadWarp) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 ::"r"(su32(tslot)), "r"(kTmCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  if (threadIdx.x == 0) {
    for (int s = 0; s < kTmStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], kTmWinWarps + g.R);  // window warps + one commit per issuer
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&wfull[b], kTmWinWarps);
      mbar_init(&wempty[b], g.R);
      mbar_init(&afull[b], g.R);
      mbar_init(&aempty[b], 4);
    }
    for (int i = 0; i < kTmIssuers; ++i) mbar_init(&drain[i], 1);
    *abort = 0;
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;
  const uint32_t acc0 = tmem, win0 = tmem + (uint32_t)g.na * g.acc_cols;

  if (warp == kTmLoadWarp) {
    // ---- loads
    if (lane == 0) {
      uint32_t q = 0;
      bool ok = true;
      for (int item = blockIdx.x; item < g.items && ok; item += gridDim.x) {
        const TmItem it = tm_item(g, item, BN);
        for (int u = 0; u < nunits; ++u, ++q) {
          const int cc = u / 3, dz = u - 3 * (u / 3);
          const int s = (int)(q % kTmStages);
          if (!tm_wait(&empty[s], ((q / kTmStages) & 1) ^ 1, abort, a.err)) {
            ok = false;
            break;
          }
          unsigned char* st = base + s * g.stage;
          const bool fullres = cc * 16 < a.c1;
          mbar_arrive_expect_tx(&full[s], fullres ? g.tx1 : g.tx2);
          if (fullres)
            tma_load_4d(st, &m1, cc * 16, it.x0 - 1, it.y0 - 1, it.z + dz - 1, &full[s]);
          else
            tma_load_4d(st, &m2, cc * 16 - a.c1, (it.x0 - 1) >> 1, (it.y0 - 1) >> 1,
                        (it.z + dz - 1) >> 1, &full[s]);
          tma_load_4d(st + g.wofs, &mw, cc * 16, it.co0, dz * 9, 0, &full[s]);
          tma_load_4d(st + g.wofs + 9 * BN * 16, &mw, cc * 16 + 8, it.co0, dz * 9, 0, &full[s]);
        }
      }
      // the copies of the last stages have landed before the block exits
      const uint32_t n = q < (uint32_t)kTmStages ? q : (uint32_t)kTmStages;
      for (uint32_t k = q - n; k < q; ++k)
        mbar_wait_bounded(&full[k % kTmStages], (k / kTmStages) & 1, a.err, kTmWaitLimit);
    }
    __syncwarp();
  } else if (warp >= kTmIssueWarp) {
    // ---- MMA issue: issuer i accumulates MMA tile i of every item
    const int i = warp - kTmIssueWarp;
    if (lane == 0 && i < g.R) {
      constexpr uint32_t kIdesc = tc_idesc(128, BN);
      uint32_t q = 0, j = 0;
      bool ok = true;
      for (int item = blockIdx.x; item < g.items && ok; item += gridDim.x, ++j) {
        const uint32_t ab = j % (uint32_t)g.na;
        if (!tm_wait(&aempty[ab], ((j / g.na) & 1) ^ 1, abort, a.err)) break;
        tc_fence_after();
        const uint32_t acc = acc0 + ab * g.acc_cols + (uint32_t)(i * BN);
        const uint32_t wrow = (uint32_t)(i * g.ty);
        for (int u = 0; u < nunits; ++u, ++q) {
          const int s = (int)(q % kTmStages);
          const uint32_t b = q & 1;
          if (!tm_wait(&full[s], (q / kTmStages) & 1, abort, a.err) ||
              !tm_wait(&wfull[b], (q >> 1) & 1, abort, a.err)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t sw = su32(base + s * g.stage + g.wofs);
          const uint32_t win = win0 + b * g.win_cols + wrow * 24;
#pragma unroll
          for (int t9 = 0; t9 < 9; ++t9) {
            const int dy = t9 / 3, dx = t9 % 3;
            tc_mma_ts(acc, win + (uint32_t)((dy * 3 + dx) * 8),
                      tc_sdesc(sw + (uint32_t)(t9 * BN * 16), 9 * BN * 16), kIdesc,
                      (u | t9) != 0 ? 1u : 0u);
          }
          tc_commit(&wempty[b]);
          tc_commit(&empty[s]);
        }
        if (!ok) break;
        tc_commit(&afull[ab]);
      }
      // every MMA this thread issued has finished before the TMEM is freed
      tc_commit(&drain[i]);
      mbar_wait_bounded(&drain[i], 0, a.err, kTmWaitLimit);
    }
    __syncwarp();
  } else if (warp >= 4) {
    // ---- windows: TMEM lane m = MMA row m = voxel (row m / tx, column m % tx);
    // two warps per lane quarter take alternate window rows
    const int quarter = warp & 3, part = (warp - 4) >> 2;
    const int m = quarter * 32 + lane;
    const int tr = m / g.tx, tc = m - tr * g.tx;
    const uint32_t lane_addr = (uint32_t)(quarter * 32) << 16;
    uint32_t q = 0;
    for (int item = blockIdx.x; item < g.items; item += gridDim.x) {
      const TmItem it = tm_item(g, item, BN);
      bool ok = true;
      for (int u = 0; u < nunits; ++u, ++q) {
        const int cc = u / 3;
        const int s = (int)(q % kTmStages);
        const uint32_t b = q & 1;
        bool w = tm_wait(&full[s], (q / kTmStages) & 1, abort, a.err);
        w = w && tm_wait(&wempty[b], ((q >> 1) & 1) ^ 1, abort, a.err);
        if (!__all_sync(kFull, w)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const unsigned char* st = base + s * g.stage;
        const bool fullres = cc * 16 < a.c1;
        const uint32_t win = lane_addr + win0 + b * g.win_cols;
#pragma unroll 1
        for (int sr = part; sr < g.S; sr += 2) {
          const int hr = sr + tr;
          uint32_t c[8], e[8], w0[8], w2[8];
          tm_slab(st, g, fullres, it.y0, it.x0, hr, tc + 1, c);
          // the warp's edge lanes fetch the neighbour outside the warp
          tm_slab(st, g, fullres, it.y0, it.x0, hr, lane == 0 ? tc : tc + 2, e);
#pragma unroll
          for (int k = 0; k < 8; ++k) {
            w0[k] = __shfl_up_sync(kFull, c[k], 1);
            w2[k] = __shfl_down_sync(kFull, c[k], 1);
            if (lane == 0) w0[k] = e[k];
            if (lane == 31) w2[k] = e[k];
          }
          const uint32_t col = win + (uint32_t)(sr * 3 * 8);
          tc_st8(col, w0);
          tc_st8(col + 8, c);
          tc_st8(col + 16, w2);
        }
        tc_wait_st();
        tc_fence_before();
        __syncwarp();
        if (lane == 0) {
          tm_arrive(&wfull[b]);
          tm_arrive(&empty[s]);
        }
      }
      if (!ok) break;
    }
  } else {
    // ---- epilogue: thread m reads TMEM lane m
    const int m = threadIdx.x;
    const int tr = m / g.tx, tc = m - tr * g.tx;
    const uint32_t lane_addr = (uint32_t)(warp * 32) << 16;
    uint32_t j = 0;
    for (int item = blockIdx.x; item < g.items; item += gridDim.x, ++j) {
      const TmItem it = tm_item(g, item, BN);
      const uint32_t ab = j % (uint32_t)g.na;
      if (!__all_sync(kFull, tm_wait(&afull[ab], (j / g.na) & 1, abort, a.err))) break;
      tc_fence_after();
      const uint32_t acc = lane_addr + acc0 + ab * g.acc_cols;
      for (int i = 0; i < g.R; ++i) {
        const int y = it.y0 + i * g.ty + tr, x = it.x0 + tc;
        const size_t o0 = (((size_t)it.z * a.H + y) * a.W + x) * a.cout + it.co0;
#pragma unroll
        for (int c0 = 0; c0 < BN; c0 += 16) {
          uint32_t r[16];
          tc_ld16(acc + (uint32_t)(i * BN + c0), r);
          uint32_t mk[8];
          if (a.mask) {
            const uint4 m0 = *reinterpret_cast<const uint4*>(a.mask + o0 + c0);
            const uint4 m1v = *reinterpret_cast<const uint4*>(a.mask + o0 + c0 + 8);
            mk[0] = m0.x; mk[1] = m0.y; mk[2] = m0.z; mk[3] = m0.w;
            mk[4] = m1v.x; mk[5] = m1v.y; mk[6] = m1v.z; mk[7] = m1v.w;
          }
          uint32_t pk[8];
#pragma unroll
          for (int k = 0; k < 8; ++k) {
            const int co = it.co0 + c0 + 2 * k;
            float v0 = __uint_as_float(r[2 * k]), v1 = __uint_as_float(r[2 * k + 1]);
            if (a.bias) {
              v0 += a.bias[co];
              v1 += a.bias[co + 1];
            }
            if (a.relu) {
              v0 = fmaxf(v0, 0.f);
              v1 = fmaxf(v1, 0.f);
            }
            if (a.mask) {
              __nv_bfloat162 mb;
              memcpy(&mb, &mk[k], 4);
              if (!(__bfloat162float(mb.x) > 0.f)) v0 = 0.f;
              if (!(__bfloat162float(mb.y) > 0.f)) v1 = 0.f;
            }
            const __nv_bfloat162 o = __floats2bfloat162_rn(v0, v1);
            memcpy(&pk[k], &o, 4);
          }
          *reinterpret_cast<uint4*>(a.y + o0 + c0) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
          *reinterpret_cast<uint4*>(a.y + o0 + c0 + 8) = make_uint4(pk[4], pk[5], pk[6], pk[7]);
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) tm_arrive(&aempty[ab]);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == kTmLoadWarp)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(kTmCols));
}
#endif

// dW[co][tap][ci] += sum over this block's voxels of dy[v][co] in(v + tap)[ci]
// (FP32 atomics; the caller zeroes dW).  GEMM M = cout (BM rows per block),
// N = 27 cin (64 columns per block: four 16-channel groups, each one tap),
// K = voxels (16 per step, kVoxChunk per block).  Warp w owns columns
// [16w, 16w + 16) of the block for all BM rows.
constexpr int kVoxChunk = 2048;
constexpr int kWRow = 72;  // smem pitch (bf16) of the [voxel][64] tiles: conflict-free

template <int BM>
__global__ void __launch_bounds__(128) k_conv3_wgrad(const Conv3Args a, const bf16* __restrict__ dy,
                                                    float* __restrict__ dw) {
  static_assert(BM % 16 == 0 && BM <= 64, "BM: 16, 32, 48 or 64");
  __shared__ alignas(128) bf16 As[2][16 * kWRow];  // [voxel][co]
  __shared__ alignas(128) bf16 Bs[2][16 * kWRow];  // [voxel][n]
  const int cin = a.c1 + a.c2;
  const int ngroups = 27 * (cin / 16);
  const int N = 27 * cin;
  const long long V = (long long)a.D * a.H * a.W;
  const int nb = blockIdx.x;           // 64-column block
  const int co0 = blockIdx.y * BM;
  const long long vbeg = (long long)blockIdx.z * kVoxChunk;
  const long long vend = vbeg + kVoxChunk < V ? vbeg + kVoxChunk : V;
  const int nsteps = (int)((vend - vbeg + 15) / 16);

  auto load = [&](int s, int stage) {
    const long long vb = vbeg + (long long)s * 16;
    // A: 16 voxels x BM channels of dy, BM/8 chunks per voxel
    for (int q = threadIdx.x; q < 16 * (BM / 8); q += CLARITY_BLOCK_STRIDE(128)) {
      const int r = q / (BM / 8), ch = q - r * (BM / 8);
      const long long v = vb + r;
      const bf16* src = v < vend ? dy + ((size_t)v * a.cout + co0 + ch * 8) : nullptr;
      cp16(&As[stage][r * kWRow + ch * 8], src, dy);
    }
    // B: 16 voxels x 4 groups x 2 halves of the shifted input
    for (int q = threadIdx.x; q < 16 * 8; q += CLARITY_BLOCK_STRIDE(128)) {
      const int r = q >> 3, gi = (q >> 1) & 3, half = q & 1;
      const int gg = nb * 4 + gi;
      const long long v = vb + r;
      const bf16* src = nullptr;
      if (v < vend && gg < ngroups) {
        const int t = gg / (cin / 16), cc = gg - t * (cin / 16);
        int dz, dyo, dx;
        tap_offset(t, &dz, &dyo, &dx);
        const int x = (int)(v % a.W);
        const long long zy = v / a.W;
        const int y = (int)(zy % a.H), z = (int)(zy / a.H);
        src = in_chunk(a, z + dz, y + dyo, x + dx, cc * 16 + half * 8);
      }
      cp16(&Bs[stage][r * kWRow + gi * 16 + half * 8], src, a.x1);
    }
    cp_commit();
  };

#ifndef CLARITY_HOST_EMULATION
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float acc[BM / 16][2][4];
#pragma unroll
  for (int i = 0; i < BM / 16; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.f;
  if (nsteps > 0) load(0, 0);
  for (int s = 0; s < nsteps; ++s) {
    const int st = s & 1;
    if (s + 1 < nsteps) {
      load(s + 1, st ^ 1);
      cp_wait<1>();
    } else {
      cp_wait<0>();
    }
    __syncthreads();
    // B fragments of the warp's two n8 tiles: stored [k][n], transposed load
    uint32_t bfr[4];
    ldm_x4_t(bfr, &Bs[st][((lane & 7) + ((lane >> 3) & 1) * 8) * kWRow + warp * 16 + (lane >> 4) * 8]);
#pragma unroll
    for (int i = 0; i < BM / 16; ++i) {
      // A fragment (rows co, cols voxel) from the stored [voxel][co] tile
      uint32_t af[4];
      ldm_x4_t(af, &As[st][((lane & 7) + (lane >> 4) * 8) * kWRow + i * 16 + ((lane >> 3) & 1) * 8]);
      mma16816(acc[i][0], af, bfr);
      mma16816(acc[i][1], af, bfr + 2);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < BM / 16; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int co = co0 + i * 16 + (lane >> 2) + h * 8;
        const int nl = warp * 16 + j * 8 + (lane & 3) * 2;  // column in the block
        const int gg = nb * 4 + (nl >> 4);
        if (gg >= ngroups) continue;
        const int n = nb * 64 + nl;
        atomicAdd(&dw[(size_t)co * N + n], acc[i][j][2 * h]);
        atomicAdd(&dw[(size_t)co * N + n + 1], acc[i][j][2 * h + 1]);
      }
#else
  static thread_local float accs[64][64];
  for (int m = 0; m < BM; ++m)
    for (int n = 0; n < 64; ++n) accs[m][n] = 0.f;
  for (int s = 0; s < nsteps; ++s) {
    load(s, 0);
    for (int m = 0; m < BM; ++m)
      for (int n = 0; n < 64; ++n) {
        float t = 0.f;
        for (int k = 0; k < 16; ++k)
          t += __bfloat162float(As[0][k * kWRow + m]) * __bfloat162float(Bs[0][k * kWRow + n]);
        accs[m][n] += t;
      }
  }
  for (int m = 0; m < BM; ++m)
    for (int n = 0; n < 64; ++n) {
      const int gg = nb * 4 + (n >> 4);
      if (gg >= ngroups) continue;
      dw[(size_t)(co0 + m) * N + nb * 64 + n] += accs[m][n];
    }
#endif
}

// ------------------------------------------------------------- SIMT kernels
// Input layer: y[v][co] = relu(b[co] + sum_tap w[co][tap] x(v + tap)), 16 outputs.
__global__ void k_conv_in(const float* __restrict__ x, int D, int H, int W,
                          const float* __restrict__ w, const float* __restrict__ b,
                          bf16* __restrict__ y) {
  __shared__ float ws[16 * 27 + 16];
  for (int i = threadIdx.x; i < 16 * 27; i += blockDim.x) ws[i] = w[i];
  for (int i = threadIdx.x; i < 16; i += blockDim.x) ws[16 * 27 + i] = b[i];
  __syncthreads();
  const long long V = (long long)D * H * W;
  for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < V;
       v += (long long)gridDim.x * blockDim.x) {
    const int xx = (int)(v % W);
    const long long zy = v / W;
    const int yy = (int)(zy % H), zz = (int)(zy / H);
    float in[27];
    for (int t = 0; t < 27; ++t) {
      int dz, dy, dx;
      tap_offset(t, &dz, &dy, &dx);
      const int z2 = zz + dz, y2 = yy + dy, x2 = xx + dx;
      in[t] = (z2 < 0 || y2 < 0 || x2 < 0 || z2 >= D || y2 >= H || x2 >= W)
                  ? 0.f
                  : x[((long long)z2 * H + y2) * W + x2];
    }
    for (int co = 0; co < 16; co += 2) {
      float r0 = ws[16 * 27 + co], r1 = ws[16 * 27 + co + 1];
      for (int t = 0; t < 27; ++t) {
        r0 += ws[co * 27 + t] * in[t];
        r1 += ws[(co + 1) * 27 + t] * in[t];
      }
      *reinterpret_cast<__nv_bfloat162*>(y + v * 16 + co) =
          __floats2bfloat162_rn(fmaxf(r0, 0.f), fmaxf(r1, 0.f));
    }
  }
}

// Input-layer gradients: dw[co][tap] += sum_v dy[v][co] x(v + tap), db[co] +=
// sum_v dy[v][co] (dy already masked by the ReLU derivative).
__global__ void k_conv_in_wgrad(const float* __restrict__ x, int D, int H, int W,
                                const bf16* __restrict__ dy, float* __restrict__ dw,
                                float* __restrict__ db) {
  __shared__ float red[16 * 28];
  for (int i = threadIdx.x; i < 16 * 28; i += blockDim.x) red[i] = 0.f;
  __syncthreads();
  float acc[16 * 28 / 16];  // each thread accumulates one output channel's 28 sums
  const int co = threadIdx.x & 15;
  for (int i = 0; i < 28; ++i) acc[i] = 0.f;
  const long long V = (long long)D * H * W;
  for (long long v = blockIdx.x * (long long)(blockDim.x / 16) + (threadIdx.x >> 4); v < V;
       v += (long long)gridDim.x * (blockDim.x / 16)) {
    const float g = __bfloat162float(dy[v * 16 + co]);
    if (g == 0.f) continue;
    const int xx = (int)(v % W);
    const long long zy = v / W;
    const int yy = (int)(zy % H), zz = (int)(zy / H);
    for (int t = 0; t < 27; ++t) {
      int dz, dyo, dx;
      tap_offset(t, &dz, &dyo, &dx);
      const int z2 = zz + dz, y2 = yy + dyo, x2 = xx + dx;
      if (z2 < 0 || y2 < 0 || x2 < 0 || z2 >= D || y2 >= H || x2 >= W) continue;
      acc[t] += g * x[((long long)z2 * H + y2) * W + x2];
    }
    acc[27] += g;
  }
  for (int i = 0; i < 28; ++i) atomicAdd(&red[co * 28 + i], acc[i]);
  __syncthreads();
  for (int i = threadIdx.x; i < 16 * 28; i += blockDim.x) {
    const int c = i / 28, k = i - c * 28;
    if (k < 27) atomicAdd(&dw[c * 27 + k], red[i]);
    else atomicAdd(&db[c], red[i]);
  }
}

// Head: r[v] = b + sum_c w[c] y[v][c] (16 channels).
__global__ void k_head(const bf16* __restrict__ y, long long V, const float* __restrict__ w,
                       const float* __restrict__ b, float* __restrict__ r) {
  for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < V;
       v += (long long)gridDim.x * blockDim.x) {
    float s = b[0];
    for (int c = 0; c < 16; ++c) s += w[c] * __bfloat162float(y[v * 16 + c]);
    r[v] = s;
  }
}

// Loss L = sum_v (r - t)^2 / V and its gradients: dy[v][c] = dL/dr w[c] masked
// by y > 0 (the last ReLU), dw[c] += sum dL/dr y[v][c], db += sum dL/dr;
// loss partial sums (FP64) into *loss by atomics.
__global__ void k_head_loss_grad(const bf16* __restrict__ y, long long V,
                                 const float* __restrict__ w, const float* __restrict__ r,
                                 const float* __restrict__ t, bf16* __restrict__ dy,
                                 float* __restrict__ dw, float* __restrict__ db,
                                 double* __restrict__ loss) {
  float gw[16];
  for (int c = 0; c < 16; ++c) gw[c] = 0.f;
  float gb = 0.f;
  double l = 0;
  const float inv = 1.f / (float)V;
  for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < V;
       v += (long long)gridDim.x * blockDim.x) {
    const float e = r[v] - t[v];
    l += (double)e * e;
    const float g = 2.f * e * inv;
    gb += g;
    for (int c = 0; c < 16; c += 2) {
      const float y0 = __bfloat162float(y[v * 16 + c]), y1 = __bfloat162float(y[v * 16 + c + 1]);
      gw[c] += g * y0;
      gw[c + 1] += g * y1;
      *reinterpret_cast<__nv_bfloat162*>(dy + v * 16 + c) =
          __floats2bfloat162_rn(y0 > 0.f ? g * w[c] : 0.f, y1 > 0.f ? g * w[c + 1] : 0.f);
    }
  }
  for (int c = 0; c < 16; ++c) atomicAdd(&dw[c], gw[c]);
  atomicAdd(db, gb);
  atomicAdd(loss, l / (double)V);
}

// Average pool 2x2x2: y[u][c] = mean of the 8 children (dims even).
__global__ void k_pool2(const bf16* __restrict__ x, int C, int D, int H, int W,
                        bf16* __restrict__ y) {
  const int D2 = D / 2, H2 = H / 2, W2 = W / 2;
  const long long n = (long long)D2 * H2 * W2 * C;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(i % C);
    const long long u = i / C;
    const int x2 = (int)(u % W2);
    const long long zy = u / W2;
    const int y2 = (int)(zy % H2), z2 = (int)(zy / H2);
    float s = 0.f;
    for (int k = 0; k < 8; ++k) {
      const int z = 2 * z2 + (k >> 2), y = 2 * y2 + ((k >> 1) & 1), xx = 2 * x2 + (k & 1);
      s += __bfloat162float(x[((long long)(z * H + y) * W + xx) * C + c]);
    }
    y[i] = __float2bfloat16_rn(0.125f * s);
  }
}

// Gradient of a skip tensor s (ReLU output, c channels): (dxcat[v][0..c) if
// given + dp[parent(v)][c] / 8) * (s > 0).  dxcat has ccat channels.
__global__ void k_merge_skip_grad(const bf16* __restrict__ dxcat, int ccat,
                                  const bf16* __restrict__ dp, const bf16* __restrict__ s,
                                  int c, int D, int H, int W, bf16* __restrict__ out) {
  const long long n = (long long)D * H * W * c;
  const int D2 = D / 2, H2 = H / 2, W2 = W / 2;
  (void)D2;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int ch = (int)(i % c);
    const long long v = i / c;
    float g = dxcat ? __bfloat162float(dxcat[v * ccat + ch]) : 0.f;
    if (dp) {
      const int xx = (int)(v % W);
      const long long zy = v / W;
      const int yy = (int)(zy % H), zz = (int)(zy / H);
      const long long u = ((long long)(zz >> 1) * H2 + (yy >> 1)) * W2 + (xx >> 1);
      g += 0.125f * __bfloat162float(dp[u * c + ch]);
    }
    out[i] = __float2bfloat16_rn(__bfloat162float(s[i]) > 0.f ? g : 0.f);
  }
}

// Gradient of the coarse (half-resolution, ReLU output) tensor read through
// nearest upsampling: sum over the 8 children of dxcat[child][c1 + c], masked
// by coarse > 0.  (D, H, W): full-resolution dims.
__global__ void k_up_grad(const bf16* __restrict__ dxcat, int ccat, int c1, int c2,
                          const bf16* __restrict__ coarse, int D, int H, int W,
                          bf16* __restrict__ out) {
  const int D2 = D / 2, H2 = H / 2, W2 = W / 2;
  const long long n = (long long)D2 * H2 * W2 * c2;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(i % c2);
    const long long u = i / c2;
    const int x2 = (int)(u % W2);
    const long long zy = u / W2;
    const int y2 = (int)(zy % H2), z2 = (int)(zy / H2);
    float s = 0.f;
    for (int k = 0; k < 8; ++k) {
      const int z = 2 * z2 + (k >> 2), y = 2 * y2 + ((k >> 1) & 1), xx = 2 * x2 + (k & 1);
      s += __bfloat162float(dxcat[((long long)(z * H + y) * W + xx) * ccat + c1 + c]);
    }
    out[i] = __float2bfloat16_rn(__bfloat162float(coarse[i]) > 0.f ? s : 0.f);
  }
}

// db[co] += sum_v dy[v][co]
__global__ void k_bias_grad(const bf16* __restrict__ dy, long long V, int cout,
                            float* __restrict__ db) {
  CLARITY_DYN_SMEM(float, sb);
  for (int i = threadIdx.x; i < cout; i += blockDim.x) sb[i] = 0.f;
  __syncthreads();
  const long long n = V * cout;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    atomicAdd(&sb[i % cout], __bfloat162float(dy[i]));
  __syncthreads();
  for (int i = threadIdx.x; i < cout; i += blockDim.x) atomicAdd(&db[i], sb[i]);
}

// Adam (Kingma and Ba, 2015) on FP32 parameters, bias-corrected.
__global__ void k_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, long long n, float lr, float b1, float b2, float eps,
                       float c1, float c2) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

// BF16 weights of one layer from its FP32 master copy [co][27][ci]: the
// forward layout and the backward-data layout wb[ci][26 - tap][co] (mirrored
// taps, transposed channels).
__global__ void k_pack_weights(const float* __restrict__ w, int cout, int cin,
                               bf16* __restrict__ wf, bf16* __restrict__ wb) {
  const long long n = (long long)cout * 27 * cin;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int ci = (int)(i % cin);
    const long long r = i / cin;
    const int t = (int)(r % 27), co = (int)(r / 27);
    const bf16 b = __float2bfloat16_rn(w[i]);
    wf[i] = b;
    if (wb) wb[((long long)ci * 27 + (26 - t)) * cout + co] = b;
  }
}

inline int grid_for(long long n, int threads = 256) {
  long long g = (n + threads - 1) / threads;
  if (g > 148 * 16) g = 148 * 16;
  return (int)(g < 1 ? 1 : g);
}

}  // namespace nn
}  // namespace clarity

// ==================================================================== C ABI
using clarity::nn::bf16;
namespace nnk = clarity::nn;

static int nn_err(cudaError_t e) {
  if (e == cudaSuccess) return CLARITY_SUCCESS;
  clarity::set_last_error(cudaGetErrorString(e));
  return e == cudaErrorMemoryAllocation ? CLARITY_DEVICE_OUT_OF_MEMORY : CLARITY_INVALID_OPERATION;
}
// The tcgen05 convolution for widths that are multiples of 32: on unless
// CLARITY_NN_TCGEN05=0, which selects the mma.sync kernel everywhere;
// CLARITY_NN_TCGEN05=require makes a call that cannot take it an error.
enum NnTcMode { kNnTcOff = 0, kNnTcOn = 1, kNnTcRequire = 2 };
static NnTcMode nn_tcgen05_mode() {
  static const NnTcMode mode = [] {
    const char* v = std::getenv("CLARITY_NN_TCGEN05");
    if (v && v[0] == '0') return kNnTcOff;
    if (v && std::strcmp(v, "require") == 0) return kNnTcRequire;
    return kNnTcOn;
  }();
  return mode;
}
static int nn_bad(const char* m) {
  clarity::set_last_error(m);
  return CLARITY_INVALID_ARGUMENT;
}

#ifndef CLARITY_HOST_EMULATION
// Geometry of the tcgen05 convolution for one call, or false when the shape
// does not suit it (width not a multiple of 32, rows not divisible).
static bool tm_geometry(const nnk::Conv3Args& a, int* bn_out, nnk::TmGeom* g, int* smem) {
  const int W = a.W, H = a.H, cout = a.cout;
  if (W % 32) return false;
  const int tx = W % 128 == 0 ? 128 : (W % 64 == 0 ? 64 : 32), ty = 128 / tx;
  const int bn = cout % 128 == 0 ? 128
                 : cout % 64 == 0 ? 64
                 : cout % 48 == 0 ? 48
                 : cout % 32 == 0 ? 32
                                  : 16;
  // the most MMA tiles per item (at most 4 rows; one issuing thread each)
  // whose accumulators and two window buffers fit the 512 TMEM columns, then
  // two accumulator buffers if they fit
  int R = 0, na = 0;
  for (int r = 4; r >= 1 && !R; r /= 2)
    for (int n = 2; n >= 1 && !R; --n) {
      if (r * ty > 4 || H % (r * ty)) continue;
      const int S = (r - 1) * ty + 3;
      if (n * r * bn + 2 * 24 * S <= nnk::kTmCols) {
        R = r;
        na = n;
      }
    }
  if (!R) return false;
  const int rows = R * ty;
  nnk::TmGeom& G = *g;
  G.tx = tx;
  G.ty = ty;
  G.R = R;
  G.rows = rows;
  G.S = (R - 1) * ty + 3;
  G.nxb = W / tx;
  G.nyb = H / rows;
  G.nnb = cout / bn;
  const long long items = (long long)G.nxb * G.nyb * a.D * G.nnb;
  if (items > 0x7fffffffll) return false;
  G.items = (int)items;
  G.na = na;
  G.cw1 = tx + 2;
  G.cw2 = tx / 2 + 2;
  const uint32_t halo1 = (uint32_t)((tx + 2) * (rows + 2) * 32);
  const uint32_t halo2 = (uint32_t)((tx / 2 + 2) * (rows / 2 + 2) * 32);
  const uint32_t wb = (uint32_t)(2 * 9 * bn * 16);
  G.wofs = (halo1 + 1023) / 1024 * 1024;
  G.stage = G.wofs + (wb + 1023) / 1024 * 1024;
  G.tx1 = halo1 + wb;
  G.tx2 = halo2 + wb;
  G.acc_cols = (uint32_t)(R * bn);
  G.win_cols = (uint32_t)(24 * G.S);
  // stages, barriers, alignment slack; at least 120 KB so one block holds an SM
  // (and its 512 TMEM columns) at a time
  int bytes = nnk::kTmStages * (int)G.stage + 512 + 1024;
  if (bytes < 120 * 1024) bytes = 120 * 1024;
  if (bytes > 227 * 1024) return false;
  *smem = bytes;
  *bn_out = bn;
  return true;
}

static int tm_sm_count() {
  int dev = 0, n = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0)
    return 148;
  return n;
}

// Launches the tcgen05 convolution.  Returns -1 when the call does not suit
// it (the caller then takes the mma.sync kernel), else a ClarityResult_t.
static int tm_conv3(const nnk::Conv3Args& a, cudaStream_t st) {
  int bn = 0, smem = 0;
  nnk::TmGeom g{};
  if (!tm_geometry(a, &bn, &g, &smem)) return -1;
  using ull = unsigned long long;
  const int cin = a.c1 + a.c2;
  clarity::TensorMap m1, m2, mw;
  {
    const ull dim[4] = {(ull)a.c1, (ull)a.W, (ull)a.H, (ull)a.D};
    const ull str[3] = {(ull)a.c1 * 2, (ull)a.W * a.c1 * 2, (ull)a.H * a.W * a.c1 * 2};
    const unsigned box[4] = {16u, (unsigned)(g.tx + 2), (unsigned)(g.rows + 2), 1u};
    if (!clarity::encode_tensor_bf16_4d(&m1, a.x1, dim, str, box, true)) return -1;
  }
  if (a.c2) {
    const ull dim[4] = {(ull)a.c2, (ull)a.W2, (ull)a.H2, (ull)a.D2};
    const ull str[3] = {(ull)a.c2 * 2, (ull)a.W2 * a.c2 * 2, (ull)a.H2 * a.W2 * a.c2 * 2};
    const unsigned box[4] = {16u, (unsigned)(g.tx / 2 + 2), (unsigned)(g.rows / 2 + 2), 1u};
    if (!clarity::encode_tensor_bf16_4d(&m2, a.x2, dim, str, box, true)) return -1;
  } else {
    m2 = m1;
  }
  {
    // weights [co][27][ci] seen as (ci, co, tap): one box is 8 channels of
    // BN outputs for 9 taps, landing as 9 tap blocks of BN 16-byte rows
    const ull dim[4] = {(ull)cin, (ull)a.cout, 27ull, 1ull};
    const ull str[3] = {27ull * cin * 2, (ull)cin * 2, 27ull * cin * a.cout * 2};
    const unsigned box[4] = {8u, (unsigned)bn, 9u, 1u};
    if (!clarity::encode_tensor_bf16_4d(&mw, a.w, dim, str, box, false)) return -1;
  }
  const int sms = tm_sm_count();
  const dim3 grid((unsigned)(g.items < sms ? g.items : sms));
  cudaError_t e = cudaSuccess;
  clarity::note_launch_begin(clarity::KK_OTHER, st);
  switch (bn) {
#define NN_TM_CASE(B)                                                                        \
  case B:                                                                                    \
    e = clarity::smem_opt_in(reinterpret_cast<const void*>(nnk::k_conv3_tm<B>), smem);      \
    if (e == cudaSuccess)                                                                    \
      CLARITY_LAUNCH(nnk::k_conv3_tm<B>, grid, nnk::kTmThreads, smem, st)(a, g, m1, m2, mw); \
    break;
    NN_TM_CASE(128)
    NN_TM_CASE(64)
    NN_TM_CASE(48)
    NN_TM_CASE(32)
    NN_TM_CASE(16)
#undef NN_TM_CASE
  }
  clarity::note_launch_end(clarity::KK_OTHER, st);
  if (e != cudaSuccess) return nn_err(e);
  return nn_err(cudaGetLastError());
}
#endif

extern "C" {

CLARITY_API ClarityResult_t clarityx_nn_conv3(const void* x1, int c1, const void* x2, int c2,
                                              int D, int H, int W, const void* w,
                                              const float* bias, int cout, int relu,
                                              const void* mask, void* y, void* stream) {
  if (!x1 || !w || !y || D <= 0 || H <= 0 || W <= 0) return (ClarityResult_t)nn_bad("conv3: argument");
  if (c1 <= 0 || c1 % 16 || c2 < 0 || c2 % 16 || (c2 && !x2) || cout <= 0 || cout % 16)
    return (ClarityResult_t)nn_bad("conv3: channel counts must be multiples of 16");
  if (c2 && (D % 2 || H % 2 || W % 2)) return (ClarityResult_t)nn_bad("conv3: upsampled input needs even dims");
  if (((uintptr_t)x1 | (uintptr_t)x2 | (uintptr_t)w | (uintptr_t)y | (uintptr_t)mask) & 15)
    return (ClarityResult_t)nn_bad("conv3: buffers must be 16-byte aligned");
  nnk::Conv3Args a{static_cast<const bf16*>(x1), c1, static_cast<const bf16*>(x2), c2, D, H, W,
                   D / 2, H / 2, W / 2, static_cast<const bf16*>(w), bias, cout, relu,
                   static_cast<const bf16*>(mask), static_cast<bf16*>(y)};
  const long long tiles = (long long)((D + nnk::kTZ - 1) / nnk::kTZ) *
                          ((H + nnk::kTY - 1) / nnk::kTY) * ((W + nnk::kTX - 1) / nnk::kTX);
  if (tiles > 0x7fffffffll) return (ClarityResult_t)nn_bad("conv3: volume too large");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (clarity::Context* ctx = clarity::global_context()) a.err = ctx->err_dev();
#ifndef CLARITY_HOST_EMULATION
  if (nn_tcgen05_mode() != kNnTcOff) {
    const int r = tm_conv3(a, st);
    if (r >= 0) return (ClarityResult_t)r;
    if (nn_tcgen05_mode() == kNnTcRequire)
      return (ClarityResult_t)nn_bad("conv3: the tcgen05 kernel cannot take this call (CLARITY_NN_TCGEN05=require)");
  }
#endif
  // output channels per block: 48 KB-class shared memory (halo + 27 taps)
  const int bn = cout % 48 == 0 ? 48 : (cout % 32 == 0 ? 32 : 16);
  const dim3 grid((unsigned)tiles, cout / bn);
  clarity::note_launch_begin(clarity::KK_OTHER, st);
  cudaError_t e = cudaSuccess;
  switch (bn) {
    case 48:
      e = clarity::smem_opt_in(reinterpret_cast<const void*>(nnk::k_conv3<48>), nnk::Conv3Smem<48>::BYTES);
      if (e == cudaSuccess) CLARITY_LAUNCH(nnk::k_conv3<48>, grid, 128, nnk::Conv3Smem<48>::BYTES, st)(a);
      break;
    case 32:
      e = clarity::smem_opt_in(reinterpret_cast<const void*>(nnk::k_conv3<32>), nnk::Conv3Smem<32>::BYTES);
      if (e == cudaSuccess) CLARITY_LAUNCH(nnk::k_conv3<32>, grid, 128, nnk::Conv3Smem<32>::BYTES, st)(a);
      break;
    default:
      e = clarity::smem_opt_in(reinterpret_cast<const void*>(nnk::k_conv3<16>), nnk::Conv3Smem<16>::BYTES);
      if (e == cudaSuccess) CLARITY_LAUNCH(nnk::k_conv3<16>, grid, 128, nnk::Conv3Smem<16>::BYTES, st)(a);
      break;
  }
  clarity::note_launch_end(clarity::KK_OTHER, st);
  if (e != cudaSuccess) return (ClarityResult_t)nn_err(e);
  return (ClarityResult_t)nn_err(cudaGetLastError());
}

CLARITY_API ClarityResult_t clarityx_nn_conv3_wgrad(const void* x1, int c1, const void* x2, int c2,
                                                    int D, int H, int W, const void* dy, int cout,
                                                    float* dw, float* dbias, void* stream) {
  if (!x1 || !dy || !dw || D <= 0 || H <= 0 || W <= 0) return (ClarityResult_t)nn_bad("wgrad: argument");
  if (c1 <= 0 || c1 % 16 || c2 < 0 || c2 % 16 || (c2 && !x2) || cout <= 0 || cout % 16)
    return (ClarityResult_t)nn_bad("wgrad: channel counts must be multiples of 16");
  if (c2 && (D % 2 || H % 2 || W % 2)) return (ClarityResult_t)nn_bad("wgrad: upsampled input needs even dims");
  if (((uintptr_t)x1 | (uintptr_t)x2 | (uintptr_t)dy) & 15)
    return (ClarityResult_t)nn_bad("wgrad: buffers must be 16-byte aligned");
  nnk::Conv3Args a{static_cast<const bf16*>(x1), c1, static_cast<const bf16*>(x2), c2, D, H, W,
                   D / 2, H / 2, W / 2, nullptr, nullptr, cout, 0, nullptr, nullptr};
  const long long V = (long long)D * H * W;
  const int cin = c1 + c2;
  const int nblk = (27 * (cin / 16) + 3) / 4;
  const int bm = cout % 64 == 0 ? 64 : (cout % 48 == 0 ? 48 : (cout % 32 == 0 ? 32 : 16));
  const dim3 grid(nblk, cout / bm, (unsigned)((V + nnk::kVoxChunk - 1) / nnk::kVoxChunk));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const bf16* d = static_cast<const bf16*>(dy);
  clarity::note_launch_begin(clarity::KK_OTHER, st);
  switch (bm) {
    case 64: CLARITY_LAUNCH(nnk::k_conv3_wgrad<64>, grid, 128, 0, st)(a, d, dw); break;
    case 48: CLARITY_LAUNCH(nnk::k_conv3_wgrad<48>, grid, 128, 0, st)(a, d, dw); break;
    case 32: CLARITY_LAUNCH(nnk::k_conv3_wgrad<32>, grid, 128, 0, st)(a, d, dw); break;
    default: CLARITY_LAUNCH(nnk::k_conv3_wgrad<16>, grid, 128, 0, st)(a, d, dw); break;
  }
  if (dbias)
    CLARITY_LAUNCH(nnk::k_bias_grad, nnk::grid_for(V * cout), 256, cout * sizeof(float), st)(
        d, V, cout, dbias);
  clarity::note_launch_end(clarity::KK_OTHER, st);
  return (ClarityResult_t)nn_err(cudaGetLastError());
}

CLARITY_API ClarityResult_t clarityx_nn_conv_in(const float* x, int D, int H, int W, const float* w,
                                                const float* b, void* y, void* stream) {
  if (!x || !w || !b || !y || D <= 0 || H <= 0 || W <= 0) return (ClarityResult_t)nn_bad("conv_in: argument");
  const long long V = (long long)D * H * W;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  CLARITY_LAUNCH(nnk::k_conv_in, nnk::grid_for(V), 256, 0, st)(x, D, H, W, w, b,
                                                               static_cast<bf16*>(y));
  return (ClarityResult_t)nn_err(cudaGetLastError());
}

CLARITY_API ClarityResult_t clarityx_nn_conv_in_wgrad(const float* x, int D, int H, int W,
                                                      const void* dy, float* dw, float* db,
                                                      void* stream) {
  if (!x || !dy || !dw || !db || D <= 0 || H <= 0 || W <= 0) return (ClarityResult_t)nn_bad("conv_in_wgrad: argument");
  const long long V = (long long)D * H * W;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  CLARITY_LAUNCH(nnk::k_conv_in_wgrad, nnk::grid_for(V * 16), 256, 0, st)(
      x, D, H, W, static_cast<const bf16*>(dy), dw, db);
  return (ClarityResult_t)nn_err(cudaGetLastError());
}

CLARITY_API ClarityResult_t clarityx_nn_head(const void* y, long long V, const float* w,
                                             const float* b, float* r, void* stream) {
  if (!y || !w || !b || !r || V <= 0) return (ClarityResult_t)nn_bad("head: argument");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  CLARITY_LAUNCH(nnk::k_head, nnk::grid_for(V), 256, 0, st)(static_cast<const bf16*>(y), V, w, b, r);
  return (ClarityResult_t)nn_err(cudaGetLastError());
}

CLARITY_API ClarityResult_t clarityx_nn_head_loss_grad(const void* y, long long V, const float* w,
                                                       const float* r, const float* t, void* dy,
                                                       float* dw, float* db, double* loss,
                                                       void* stream) {
  if (!y || !w || !r || !t || !dy || !dw || !db || !loss || V <= 0)
    return (ClarityResult_t)nn_bad("head_loss_grad: argument");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  CLARITY_LAUNCH(nnk::k_head_loss_grad, nnk::grid_for(V), 256, 0, st)(
      static_cast<const bf16*>(y), V, w, r, t, static_cast<bf16*>(dy), dw, db, loss);
  return (ClarityResult_t)nn_err(cudaGetLastError());
}

CLARITY_API ClarityResult_t clarityx_nn_pool2(const void* x, int C, int D, int H, int W, void* y,
                                              void* stream) {
  if (!x || !y || C <= 0 || D <= 0 || H <= 0 || W <= 0 || D % 2 || H % 2 || W % 2)
    return (ClarityResult_t)nn_bad("pool2: argument (dims must be even)");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  CLARITY_LAUNCH(nnk::k_pool2, nnk::grid_for((long long)D * H * W * C / 8), 256, 0, st)(
      static_cast<const bf16*>(x), C, D, H, W, static_cast<bf16*>(y));
  return (ClarityResult_t)nn_err(cudaGetLastError());
}

CLARITY_API ClarityResult_t clarityx_nn_merge_skip_grad(const void* dxcat, int ccat,
                                                        const void* dp, const void* s, int c,
                                                        int D, int H, int W, void* out,
                                                        void* stream) {
  if (!s || !out || c <= 0 || D <= 0 || H <= 0 || W <= 0 || (dp && (D % 2 || H % 2 || W % 2)) ||
      (dxcat && ccat < c))
    return (ClarityResult_t)nn_bad("merge_skip_grad: argument");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  CLARITY_LAUNCH(nnk::k_merge_skip_grad, nnk::grid_for((long long)D * H * W * c), 256, 0, st)(
      static_cast<const bf16*>(dxcat), ccat, static_cast<const bf16*>(dp),
      static_cast<const bf16*>(s), c, D, H, W, static_cast<bf16*>(out));
  return (ClarityResult_t)nn_err(cudaGetLastError());
}

CLARITY_API ClarityResult_t clarityx_nn_up_grad(const void* dxcat, int ccat, int c1, int c2,
                                                const void* coarse, int D, int H, int W,
                                                void* out, void* stream) {
  if (!dxcat || !coarse || !out || c2 <= 0 || c1 < 0 || ccat != c1 + c2 || D % 2 || H % 2 ||
      W % 2 || D <= 0 || H <= 0 || W <= 0)
    return (ClarityResult_t)nn_bad("up_grad: argument");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  CLARITY_LAUNCH(nnk::k_up_grad, nnk::grid_for((long long)D * H * W * c2 / 8), 256, 0, st)(
      static_cast<const bf16*>(dxcat), ccat, c1, c2, static_cast<const bf16*>(coarse), D, H, W,
      static_cast<bf16*>(out));
  return (ClarityResult_t)nn_err(cudaGetLastError());
}

CLARITY_API ClarityResult_t clarityx_nn_adam(float* p, const float* g, float* m, float* v,
                                             long long n, float lr, float b1, float b2, float eps,
                                             int step, void* stream) {
  if (!p || !g || !m || !v || n <= 0 || step <= 0) return (ClarityResult_t)nn_bad("adam: argument");
  const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  CLARITY_LAUNCH(nnk::k_adam, nnk::grid_for(n), 256, 0, st)(p, g, m, v, n, lr, b1, b2, eps, c1, c2);
  return (ClarityResult_t)nn_err(cudaGetLastError());
}

CLARITY_API ClarityResult_t clarityx_nn_pack_weights(const float* w, int cout, int cin, void* wf,
                                                     void* wb, void* stream) {
  if (!w || !wf || cout <= 0 || cin <= 0) return (ClarityResult_t)nn_bad("pack_weights: argument");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  CLARITY_LAUNCH(nnk::k_pack_weights, nnk::grid_for((long long)cout * 27 * cin), 256, 0, st)(
      w, cout, cin, static_cast<bf16*>(wf), static_cast<bf16*>(wb));
  return (ClarityResult_t)nn_err(cudaGetLastError());
}

}  // extern "C"

// ============================================== learned start (library form)
// The network's forward pass and the learned-start solve in C++, so a C
// caller needs no Python: RL `pre` iterations, the U-Net's prediction, RL
// resumed from it.  The domain transforms around the network are fused into
// its first and last kernels: the input layer reads log(x/m + 0.01) on the
// fly, and the head writes the advanced estimate m ((x/m + 0.01) e^r - 0.01),
// clamped at 0, instead of r (m = mean(x), an FP64 device reduction).  No
// host round trip and no other kernel sits between the RL iterate and the
// resumed RL.
namespace clarity {
namespace nn {

constexpr float kDomainEps = 0.01f;

// The network's layers in the order of the FP32 parameter vector: for each,
// weights [co][27][c1 + c2] then bias [co]; then the head (16 weights, 1 bias).
// Index: 0 l0a (1 -> 16, SIMT), 1 l0b, 2 l1a, 3 l1b, 4 l2a, 5 l2b, 6 l3a,
// 7 l3b, 8 l2c (skip 64 + up 128), 9 l2d, 10 l1c (32 + 64), 11 l1d,
// 12 l0c (16 + 32), 13 l0d.
struct NetLayer {
  int c1, c2, co;
};
constexpr NetLayer kNet[14] = {{1, 0, 16},    {16, 0, 16},  {16, 0, 32},  {32, 0, 32},
                               {32, 0, 64},   {64, 0, 64},  {64, 0, 128}, {128, 0, 128},
                               {64, 128, 64}, {64, 0, 64},  {32, 64, 32}, {32, 0, 32},
                               {16, 32, 16},  {16, 0, 16}};

inline long long layer_weights(int l) {
  return (long long)kNet[l].co * 27 * (kNet[l].c1 + kNet[l].c2);
}
// Offset of layer l's weights in the parameter vector (its bias follows).
inline long long layer_offset(int l) {
  long long o = 0;
  for (int i = 0; i < l; ++i) o += layer_weights(i) + kNet[i].co;
  return o;
}

// FP64 partial sums of x, then m = max(sum / V, 1e-20) as float.
__global__ void k_nn_sum(const float* __restrict__ x, long long V, double* __restrict__ partial) {
  double acc = 0;
  for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < V;
       v += (long long)gridDim.x * blockDim.x)
    acc += (double)x[v];
  block_sum_store(acc, partial);
}
__global__ void k_nn_mean(const double* partial, int np, long long V, float* mean) {
  const double t = block_total(partial, np);
  if (threadIdx.x == 0) mean[0] = fmaxf((float)(t / (double)V), 1e-20f);
}

// Input layer on the log-domain input read on the fly: in(v) = log(x/m +
// 0.01) inside the volume, 0 outside (zero padding of the transformed
// input, as the separate transform + k_conv_in computes it).
__global__ void k_conv_in_log(const float* __restrict__ x, int D, int H, int W,
                              const float* __restrict__ w, const float* __restrict__ b,
                              const float* __restrict__ mean, bf16* __restrict__ y) {
  __shared__ float ws[16 * 27 + 16];
  for (int i = threadIdx.x; i < 16 * 27; i += blockDim.x) ws[i] = w[i];
  for (int i = threadIdx.x; i < 16; i += blockDim.x) ws[16 * 27 + i] = b[i];
  __syncthreads();
  const float m = *mean;
  const long long V = (long long)D * H * W;
  for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < V;
       v += (long long)gridDim.x * blockDim.x) {
    const int xx = (int)(v % W);
    const long long zy = v / W;
    const int yy = (int)(zy % H), zz = (int)(zy / H);
    float in[27];
    for (int t = 0; t < 27; ++t) {
      int dz, dy, dx;
      tap_offset(t, &dz, &dy, &dx);
      const int z2 = zz + dz, y2 = yy + dy, x2 = xx + dx;
      in[t] = (z2 < 0 || y2 < 0 || x2 < 0 || z2 >= D || y2 >= H || x2 >= W)
                  ? 0.f
                  : logf(x[((long long)z2 * H + y2) * W + x2] / m + kDomainEps);
    }
    for (int co = 0; co < 16; co += 2) {
      float r0 = ws[16 * 27 + co], r1 = ws[16 * 27 + co + 1];
      for (int t = 0; t < 27; ++t) {
        r0 += ws[co * 27 + t] * in[t];
        r1 += ws[(co + 1) * 27 + t] * in[t];
      }
      *reinterpret_cast<__nv_bfloat162*>(y + v * 16 + co) =
          __floats2bfloat162_rn(fmaxf(r0, 0.f), fmaxf(r1, 0.f));
    }
  }
}

// Head with the prediction: r = b + sum_c w[c] y[v][c];
// out[v] = max(0, m ((x[v]/m + 0.01) e^r - 0.01)).
__global__ void k_head_predict(const bf16* __restrict__ y, long long V, const float* __restrict__ w,
                               const float* __restrict__ b, const float* __restrict__ x,
                               const float* __restrict__ mean, float* __restrict__ out) {
  const float m = *mean;
  for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < V;
       v += (long long)gridDim.x * blockDim.x) {
    float r = b[0];
    for (int c = 0; c < 16; ++c) r += w[c] * __bfloat162float(y[v * 16 + c]);
    const float p = m * ((x[v] / m + kDomainEps) * expf(r) - kDomainEps);
    out[v] = fmaxf(p, 0.f);
  }
}

constexpr int kMeanBlocks = 592;

inline size_t round_up(size_t v) { return (v + 255) & ~size_t(255); }

}  // namespace nn

long long nn_param_count() {
  return nn::layer_offset(14) + 16 + 1;
}

#ifndef CL_CHECK
#define CL_CHECK(call)                                         \
  do {                                                         \
    cudaError_t e_ = (call);                                   \
    if (e_ != cudaSuccess) return status_from_cuda(e_, #call); \
  } while (0)
#endif
#ifndef CL_TRY
#define CL_TRY(expr)         \
  do {                       \
    Status s_ = (expr);      \
    if (!s_.ok()) return s_; \
  } while (0)
#endif

#define NN_TRY(expr)                                                   \
  do {                                                                 \
    const ClarityResult_t r_ = (expr);                                 \
    if (r_ != CLARITY_SUCCESS) {                                       \
      Status s_;                                                       \
      s_.code = r_;                                                    \
      s_.msg = std::string("network: ") + #expr;                       \
      return s_;                                                       \
    }                                                                  \
  } while (0)

Status nn_predict(Context& ctx, const float* params, const float* x, int D, int H, int W,
                  float* out) {
  using namespace nn;
  if (D % 8 || H % 8 || W % 8) {
    Status s;
    s.code = CLARITY_INVALID_ARGUMENT;
    s.msg = "learned start: volume dimensions must be multiples of 8 (three poolings)";
    return s;
  }
  const long long V = (long long)D * H * W;
  // scratch: partials | mean | BF16 weights of layers 1..13 | activations
  size_t off = 0;
  const size_t o_part = off;
  off = round_up(off + sizeof(double) * kMeanBlocks);
  const size_t o_mean = off;
  off = round_up(off + sizeof(float));
  size_t o_w[14] = {};
  for (int l = 1; l < 14; ++l) {
    o_w[l] = off;
    off = round_up(off + sizeof(bf16) * (size_t)layer_weights(l));
  }
  // activations per level: three buffers at full resolution (16 ch), three
  // at 1/2 (32 ch), three at 1/4 (64 ch), two at 1/8 (128 ch)
  const long long lv[4] = {V * 16, V / 8 * 32, V / 64 * 64, V / 512 * 128};
  const int nbuf[4] = {3, 3, 3, 2};
  size_t o_a[4][3] = {};
  for (int k = 0; k < 4; ++k)
    for (int j = 0; j < nbuf[k]; ++j) {
      o_a[k][j] = off;
      off = round_up(off + sizeof(bf16) * (size_t)lv[k]);
    }
  void* base = nullptr;
  CL_TRY(ctx.aux_scratch(off, &base));
  char* sc = static_cast<char*>(base);
  double* part = reinterpret_cast<double*>(sc + o_part);
  float* mean = reinterpret_cast<float*>(sc + o_mean);
  bf16* wf[14] = {};
  for (int l = 1; l < 14; ++l) wf[l] = reinterpret_cast<bf16*>(sc + o_w[l]);
  auto act = [&](int k, int j) { return reinterpret_cast<bf16*>(sc + o_a[k][j]); };
  cudaStream_t st = ctx.exec_stream();
  void* sv = static_cast<void*>(st);
  // BF16 forward weights from the FP32 parameters
  for (int l = 1; l < 14; ++l)
    NN_TRY(clarityx_nn_pack_weights(params + layer_offset(l), kNet[l].co,
                                    kNet[l].c1 + kNet[l].c2, wf[l], nullptr, sv));
  // m = mean(x)
  note_launch_begin(KK_OTHER, st);
  CLARITY_LAUNCH(k_nn_sum, kMeanBlocks, 256, 0, st)(x, V, part);
  CLARITY_LAUNCH(k_nn_mean, 1, 256, 0, st)(part, kMeanBlocks, V, mean);
  CLARITY_LAUNCH(k_conv_in_log, grid_for(V), 256, 0, st)(x, D, H, W, params + layer_offset(0),
                                                         params + layer_offset(0) +
                                                             layer_weights(0),
                                                         mean, act(0, 0));
  note_launch_end(KK_OTHER, st);
  CL_CHECK(cudaGetLastError());
  auto conv = [&](int l, const bf16* x1, const bf16* x2, int d, int h, int w, bf16* y) {
    return clarityx_nn_conv3(x1, kNet[l].c1, x2, kNet[l].c2, d, h, w, wf[l],
                             params + layer_offset(l) + layer_weights(l), kNet[l].co, 1,
                             nullptr, y, sv);
  };
  auto pool = [&](const bf16* a, int c, int d, int h, int w, bf16* y) {
    return clarityx_nn_pool2(a, c, d, h, w, y, sv);
  };
  const int d0 = D, h0 = H, w0 = W, d1 = D / 2, h1 = H / 2, w1 = W / 2, d2 = D / 4, h2 = H / 4,
            w2 = W / 4, d3 = D / 8, h3 = H / 8, w3 = W / 8;
  // encoder: a0 -> s0 (kept) -> p0 -> a1 -> s1 (kept) -> p1 -> a2 -> s2 (kept) -> p2
  NN_TRY(conv(1, act(0, 0), nullptr, d0, h0, w0, act(0, 1)));   // s0
  NN_TRY(pool(act(0, 1), 16, d0, h0, w0, act(1, 0)));            // p0
  NN_TRY(conv(2, act(1, 0), nullptr, d1, h1, w1, act(1, 2)));   // a1
  NN_TRY(conv(3, act(1, 2), nullptr, d1, h1, w1, act(1, 1)));   // s1
  NN_TRY(pool(act(1, 1), 32, d1, h1, w1, act(2, 0)));            // p1
  NN_TRY(conv(4, act(2, 0), nullptr, d2, h2, w2, act(2, 2)));   // a2
  NN_TRY(conv(5, act(2, 2), nullptr, d2, h2, w2, act(2, 1)));   // s2
  NN_TRY(pool(act(2, 1), 64, d2, h2, w2, act(3, 0)));            // p2
  NN_TRY(conv(6, act(3, 0), nullptr, d3, h3, w3, act(3, 1)));   // a3
  NN_TRY(conv(7, act(3, 1), nullptr, d3, h3, w3, act(3, 0)));   // b3
  // decoder: skip + nearest-upsampled coarse tensor, read inside the loader
  NN_TRY(conv(8, act(2, 1), act(3, 0), d2, h2, w2, act(2, 0)));  // c2
  NN_TRY(conv(9, act(2, 0), nullptr, d2, h2, w2, act(2, 2)));    // d2
  NN_TRY(conv(10, act(1, 1), act(2, 2), d1, h1, w1, act(1, 0))); // c1
  NN_TRY(conv(11, act(1, 0), nullptr, d1, h1, w1, act(1, 2)));   // d1
  NN_TRY(conv(12, act(0, 1), act(1, 2), d0, h0, w0, act(0, 0))); // c0
  NN_TRY(conv(13, act(0, 0), nullptr, d0, h0, w0, act(0, 2)));   // d0
  const float* head = params + layer_offset(14);
  note_launch_begin(KK_OTHER, st);
  CLARITY_LAUNCH(k_head_predict, grid_for(V), 256, 0, st)(act(0, 2), V, head, head + 16, x, mean,
                                                          out);
  note_launch_end(KK_OTHER, st);
  CL_CHECK(cudaGetLastError());
  return Status::Ok();
}

Status run_ml_learned(Context& ctx, const float* img, Dims id, const float* ker, Dims kd,
                      const float* params, int pre, float* out, int post, double* idiv) {
  if (id.x % 8 || id.y % 8 || id.z % 8) {
    Status s;
    s.code = CLARITY_INVALID_ARGUMENT;
    s.msg = "learned start: image dimensions must be multiples of 8 (three poolings)";
    return s;
  }
  if (pre < 0 || post < 0) {
    Status s;
    s.code = CLARITY_INVALID_ARGUMENT;
    s.msg = "learned start: pre and post must be >= 0";
    return s;
  }
  // the early iterate and the prediction live in the workspace's spare
  // volumes (accelerated-RL buffers, allocated on first use)
  const PlanEntry* pe;
  CL_TRY(ctx.plan(Dims{id.x + kd.x, id.y + kd.y, id.z + kd.z}, &pe));
  Workspace* ws;
  CL_TRY(ctx.workspace(*pe, id, kd, &ws));
  const long long n = id.n();
  if (ws->xbuf_cap < n) {
    for (float*& b : ws->xbuf) {
      cudaFree(b);
      b = nullptr;
    }
    ws->xbuf_cap = 0;
    for (float*& b : ws->xbuf) CL_CHECK(dev_alloc((void**)&b, sizeof(float) * (size_t)n));
    ws->xbuf_cap = n;
  }
  float* early = ws->xbuf[0];
  float* start = ws->xbuf[1];
  CL_TRY(run_rl_ex(ctx, img, id, ker, kd, nullptr, early, pre, nullptr));
  CL_TRY(nn_predict(ctx, params, early, id.z, id.y, id.x, start));
  return run_rl_ex(ctx, img, id, ker, kd, start, out, post, idiv);
}

}  // namespace clarity
