// kern_batch.cu -- Richardson-Lucy on many volumes of uneven sizes in ONE
// persistent launch (src/MaximumLikelihoodDeconvolve.cxx:48-81 per volume;
// the reference runs one volume per call).
//
// Every volume's iterations are split into passes -- z (OTF, deferred flux
// scale), xy ratio, z (OTF), xy product, flux-scale finish -- and every pass
// into tiles, the same tiles the per-volume kernels give one block each.  A
// host-built queue lists the passes in the order (volume set, iteration,
// pass, volume), so the work of a set's volumes interleaves and every pass
// comes after the one it depends on.  A fixed grid of blocks (as many as
// are resident at once) takes work items (one tile of one pass) from the
// queue with an atomic ticket; before its first item of a pass a block
// waits until every tile of the pass before it (same volume) has
// completed, then runs the tile with the pass bodies of passes.cuh and
// counts it done.  A block only ever waits for items taken earlier, by
// blocks already running, so the queue drains whatever the grid size.  The
// waits are bounded: one that runs out records a timeout in the error word
// and raises a flag at which every block stops.
//
// Data written earlier in the launch is read with ordinary loads after an
// acquire (the macros below replace the read-only-cache loads and
// __restrict__ of the pass bodies in this file only), and an item's tile
// stands in for the block index the fused operations use for their partial
// sums.
#include "launch_macro.cuh"

namespace clarity {
namespace batchk {
// the running item's tile and its pass's tile count (one block, many items)
__shared__ int s_tile;
__shared__ int s_tiles;
}  // namespace batchk
}  // namespace clarity

#undef CLARITY_BLOCK_ID
#define CLARITY_BLOCK_ID() ((unsigned)::clarity::batchk::s_tile)
#undef CLARITY_GRID_DIM
#define CLARITY_GRID_DIM() ((unsigned)::clarity::batchk::s_tiles)
#undef CLARITY_RESTRICT
#define CLARITY_RESTRICT
#undef CLARITY_LDG
#define CLARITY_LDG(p) (*(p))

#include <algorithm>
#include <cstdlib>
#include <vector>

#include "engine.hpp"
#include "ops.cuh"
#include "passes.cuh"

namespace clarity {

#define CL_CHECK(call)                                         \
  do {                                                         \
    cudaError_t e_ = (call);                                   \
    if (e_ != cudaSuccess) return status_from_cuda(e_, #call); \
  } while (0)
#define CL_TRY(expr)         \
  do {                       \
    Status s_ = (expr);      \
    if (!s_.ok()) return s_; \
  } while (0)

namespace batchk {

// Pass kinds of one RL iteration, in order.
enum : int { kZ2 = 0, kRatio = 1, kZ4 = 2, kProduct = 3, kFinish = 4, kKinds = 5 };

// One volume of the batch (device-resident table).
struct Vol {
  VolPlan P;
  const float2* tw;
  const int* xrev;
  float2* S;
  const float2* H;
  float* u;
  double* partial;
  double* dscal;  // [0] energy, [1] last sum
  float* fscal;   // [0] deferred flux scale
  int* iscal;     // [0] partials the product pass wrote
  ImageSrc g;
  WorkVol w;
  float scale_n;
  int tiles[kKinds];
};

// Queue layout.  The volumes run in sets of consecutive volumes; set j holds
// volumes [v0, v0 + nv), its items follow all of set j-1's, and within the
// set iteration k occupies [start + k*L, start + (k+1)*L), in the order
// (kind, volume) with group q = kind*nv + (v - v0) at [pre[poff + q],
// pre[poff + q + 1]) from the iteration's first item.  Pass (k, kind, v) is
// done when done[(k*kKinds + kind)*nvol + v] equals its tile count.  One set
// of all volumes interleaves every volume's passes (no waits between passes
// of one volume); smaller sets keep fewer volumes' spectra in flight, so more
// of a pass's output is still in L2 when the next pass reads it.
struct VolSet {
  long long start, L;
  int poff, v0, nv;
};
struct Queue {
  int nvol, iters, nsets;
  long long total;  // items over all sets
  int* ticket;      // [0] next item, [1] abort flag
  int* done;        // [iters * kKinds * nvol] completed tiles per pass
  int* err;
};

constexpr long long kWaitPolls = 1ll << 22;

__device__ __forceinline__ int load_acquire(const int* p) {
#ifndef CLARITY_HOST_EMULATION
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
#else
  return *p;
#endif
}
__device__ __forceinline__ void backoff() {
#ifndef CLARITY_HOST_EMULATION
  __nanosleep(128);
#endif
}

// Runs tile `tile` of pass (iteration k, kind, volume v).
__device__ __forceinline__ void run_item(float2* sm, const VolPlan& P, const Vol& V, int k,
                                         int iters, int kind, int tile) {
  const float* sk = k == 0 ? nullptr : V.fscal;  // deferred flux scale
  switch (kind) {
    case kZ2: {
      // the ratio pass reads only planes z < Z: the rest are not stored
      ModOTF m{V.H, V.scale_n, sk};
      m.zout = V.g.Z;
      z_body(sm, P, m, V.S, V.S, V.tw, tile);
      break;
    }
    case kRatio: {
      MidRLRatio r{V.g, P.xmode};
      xy_inv_fwd_body(sm, P, r, V.S, V.tw, V.xrev, tile);
      break;
    }
    case kZ4: {
      // the ratio is zero in planes z >= Z: read as zeros
      ModOTF m{V.H, V.scale_n};
      m.zn = V.g.Z;
      z_body(sm, P, m, V.S, V.S, V.tw, tile);
      break;
    }
    case kProduct: {
      EpiRLProduct e;
      e.cur = k == 0 ? nullptr : V.u;
      e.g = V.g;
      e.scale = sk;
      e.unew = V.u;
      e.partial = V.partial;
      e.w = V.w;
      e.xmode = P.xmode;
      e.acc = 0.0;
      e.nblocks = V.iscal;
      if (k + 1 < iters)
        xy_inv_fwd_body(sm, P, e, V.S, V.tw, V.xrev, tile);
      else
        xy_inverse_body(sm, P, e, V.S, V.tw, V.xrev, tile);
      break;
    }
    default: {
      // s = E / sum u' in float, in the fixed order of block_total
      const double t = block_total(V.partial, *V.iscal);
      if (threadIdx.x == 0) {
        V.dscal[1] = t;
        V.fscal[0] = (float)V.dscal[0] / (float)t;
      }
      break;
    }
  }
}

__global__ void __launch_bounds__(256, CLARITY_GEN_MINB)
    k_rl_batch(const Vol* vols, const VolSet* sets, const long long* pre, const Queue q) {
  CLARITY_DYN_SMEM(float2, sm);
  __shared__ int s_stop, s_k, s_kind, s_vol;
  __shared__ VolPlan s_plan;
  int have = -1;        // the pass whose dependency this block has seen complete
  int cached_vol = -1;  // the volume whose plan s_plan holds
  // thread 0 takes its next ticket while the block runs the current item, so
  // the atomic's round trip is hidden (a block holds at most two tickets:
  // the one it runs and the next)
  long long next = threadIdx.x == 0 ? (long long)atomicAdd(&q.ticket[0], 1) : 0;
  for (;;) {
    if (threadIdx.x == 0) {
      int stop = 0;
      const long long it = next;
      if (it < q.total) next = (long long)atomicAdd(&q.ticket[0], 1);
      int k = 0, kind = 0, v = 0;
      if (it < q.total) {
        int lo = 0, hi = q.nsets - 1;  // the set with start <= it
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if (sets[mid].start <= it) lo = mid;
          else hi = mid - 1;
        }
        const VolSet S = sets[lo];
        const long long r = it - S.start;
        k = (int)(r / S.L);
        const long long r2 = r - (long long)k * S.L;
        const long long* P = pre + S.poff;
        lo = 0;
        hi = kKinds * S.nv - 1;  // the group with P[g] <= r2 < P[g + 1]
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if (P[mid] <= r2) lo = mid;
          else hi = mid - 1;
        }
        kind = lo / S.nv;
        v = S.v0 + (lo - kind * S.nv);
        s_tile = (int)(r2 - P[lo]);
        const int pass = (k * kKinds + kind) * q.nvol + v;
        if (pass != have) {
          // the pass before: the previous kind of the same volume, or the
          // previous iteration's finish
          int dep = -1, dkind = 0;
          if (kind > 0) {
            dep = pass - q.nvol;
            dkind = kind - 1;
          } else if (k > 0) {
            dep = ((k - 1) * kKinds + kFinish) * q.nvol + v;
            dkind = kFinish;
          }
          if (dep >= 0) {
            const int need = vols[v].tiles[dkind];
            long long polls = 0;
            while (load_acquire(&q.done[dep]) < need) {
              if (load_acquire(&q.ticket[1])) {
                stop = 1;
                break;
              }
              if (++polls > kWaitPolls) {
                raise_error(q.err, kErrWaitTimeout);
                atomicExch(&q.ticket[1], 1);
                stop = 1;
                break;
              }
              backoff();
            }
            __threadfence();  // the block's later loads see the pass's writes
          }
          have = pass;
        }
      }
      s_stop = stop || it >= q.total;
      s_k = k;
      s_kind = kind;
      s_vol = v;
    }
    __syncthreads();
    if (s_stop) break;
    const int v = s_vol, kind = s_kind;
    const Vol& V = vols[v];
    // the volume's plan in shared memory for the pass bodies (consecutive
    // items are mostly of one volume: copied when the volume changes)
    if (v != cached_vol) {
      const int* src = reinterpret_cast<const int*>(&V.P);
      int* dst = reinterpret_cast<int*>(&s_plan);
      for (int i = threadIdx.x; i < (int)(sizeof(VolPlan) / sizeof(int)); i += blockDim.x)
        dst[i] = src[i];
      cached_vol = v;
    }
    if (threadIdx.x == 0) s_tiles = V.tiles[kind];
    __syncthreads();
    run_item(sm, s_plan, V, s_k, q.iters, kind, s_tile);
    // every thread's writes of this tile, then the count (release)
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      atomicAdd(&q.done[((long long)s_k * kKinds + kind) * q.nvol + v], 1);
    }
  }
}

// Words of a table carried in the kernel's parameters (a graph keeps them by
// value, so a replayed graph rewrites its own tables).
constexpr int kPutWords = 960;
struct Words {
  int n;
  unsigned w[kPutWords];
};
__global__ void k_put_words(unsigned* dst, const Words w) {
  for (int i = threadIdx.x; i < w.n; i += blockDim.x) dst[i] = w.w[i];
}

}  // namespace batchk

// The iterations of an RL batch as one persistent launch.  The volumes' OTFs,
// energies and first forward transforms are done (on `st`); this enqueues
// the queue reset, the launch and nothing else.  scratch: a device buffer of
// at least batch_queue_bytes(n, iters) bytes.
size_t batch_queue_bytes(int n, int iters) {
  const size_t vols = sizeof(batchk::Vol) * (size_t)n;
  const size_t sets = sizeof(batchk::VolSet) * (size_t)n;
  const size_t pre = sizeof(long long) * ((size_t)batchk::kKinds * n + (size_t)n);
  const size_t counters = sizeof(int) * (2 + (size_t)iters * batchk::kKinds * n);
  return ((vols + 255) & ~size_t(255)) + ((sets + 255) & ~size_t(255)) +
         ((pre + 255) & ~size_t(255)) + counters;
}

// Volumes per set of the persistent queue: CLARITY_BATCH_SET, default all.
static int batch_set_size(int n) {
  static const int v = [] {
    const char* e = std::getenv("CLARITY_BATCH_SET");
    return e ? std::atoi(e) : 0;
  }();
  return v > 0 && v < n ? v : n;
}

Status launch_rl_batch(Context& ctx, int n, const PlanEntry* const* pes, Workspace* const* wss,
                       const float* const* imgs, const Dims* ids, const Dims* wds, int iters,
                       void* scratch, cudaStream_t st) {
  using batchk::Vol;
  using batchk::VolSet;
  constexpr int K = batchk::kKinds;
  std::vector<Vol> vols(n);
  int smem = 0;
  for (int i = 0; i < n; ++i) {
    const VolPlan& P = pes[i]->P;
    Vol& V = vols[i];
    V.P = P;
    V.tw = pes[i]->tw;
    V.xrev = pes[i]->xrev;
    V.S = wss[i]->S;
    V.H = wss[i]->H;
    V.u = wss[i]->u;
    V.partial = wss[i]->partial;
    V.dscal = wss[i]->dscal;
    V.fscal = wss[i]->fscal;
    V.iscal = wss[i]->iscal;
    V.g = ImageSrc{imgs[i], ids[i].x, ids[i].y, ids[i].z};
    V.w = WorkVol{wds[i].x, wds[i].y, wds[i].z};
    V.scale_n = (float)(1.0 / ((double)wds[i].x * wds[i].y * wds[i].z));
    const int ngroups = P.By / P.G;
    V.tiles[batchk::kZ2] = P.z_blocks;
    V.tiles[batchk::kRatio] = std::min(ids[i].z, P.nz) * ngroups;  // planes z < Z only
    V.tiles[batchk::kZ4] = P.z_blocks;
    V.tiles[batchk::kProduct] = P.xy_blocks;
    V.tiles[batchk::kFinish] = 1;
    if (P.xy_threads != 256 || P.z_threads != 256) {
      Status s;
      s.code = CLARITY_INVALID_OPERATION;
      s.msg = "persistent batch: a plan with other than 256 threads per block";
      return s;
    }
    smem = std::max(smem, std::max(P.xy_smem, P.z_smem));
  }
  // the sets and, per set, the offsets of its (kind, volume) groups
  const int per = batch_set_size(n);
  std::vector<VolSet> sets;
  std::vector<long long> pre;
  long long total = 0;
  for (int v0 = 0; v0 < n; v0 += per) {
    VolSet S;
    S.v0 = v0;
    S.nv = std::min(per, n - v0);
    S.poff = (int)pre.size();
    S.start = total;
    pre.push_back(0);
    for (int kind = 0; kind < K; ++kind)
      for (int v = v0; v < v0 + S.nv; ++v) pre.push_back(pre.back() + vols[v].tiles[kind]);
    S.L = pre.back() - pre[S.poff];
    total += S.L * iters;
    sets.push_back(S);
  }
  batchk::Queue q;
  q.nvol = n;
  q.iters = iters;
  q.nsets = (int)sets.size();
  q.total = total;
  if (q.total >= (1ll << 31) || (long long)iters * K * n >= (1ll << 31)) {
    Status s;
    s.code = CLARITY_INVALID_ARGUMENT;
    s.msg = "persistent batch: more than 2^31 work items";
    return s;
  }
  unsigned char* base = static_cast<unsigned char*>(scratch);
  const size_t vb = (sizeof(Vol) * (size_t)n + 255) & ~size_t(255);
  const size_t sb = (sizeof(VolSet) * (size_t)n + 255) & ~size_t(255);
  const size_t pb = (sizeof(long long) * ((size_t)K * n + (size_t)n) + 255) & ~size_t(255);
  Vol* dvols = reinterpret_cast<Vol*>(base);
  VolSet* dsets = reinterpret_cast<VolSet*>(base + vb);
  long long* dpre = reinterpret_cast<long long*>(base + vb + sb);
  int* counters = reinterpret_cast<int*>(base + vb + sb + pb);
  q.ticket = counters;
  q.done = counters + 2;
  q.err = ctx.err_dev();
  const size_t nctr = 2 + (size_t)iters * K * n;
  // the tables travel in kernel parameters (no host buffer has to outlive a
  // captured graph), then the counters start at zero
  auto put = [&](void* dst, const void* src, size_t bytes) -> Status {
    const unsigned* w = static_cast<const unsigned*>(src);
    const size_t nw = bytes / sizeof(unsigned);
    for (size_t o = 0; o < nw; o += batchk::kPutWords) {
      batchk::Words chunk;
      chunk.n = (int)std::min<size_t>(batchk::kPutWords, nw - o);
      std::copy(w + o, w + o + chunk.n, chunk.w);
      count_launch();
      CLARITY_LAUNCH(batchk::k_put_words, 1, 256, 0, st)(static_cast<unsigned*>(dst) + o, chunk);
      CL_CHECK(cudaGetLastError());
    }
    return Status::Ok();
  };
  static_assert(sizeof(Vol) % sizeof(unsigned) == 0, "table of whole words");
  static_assert(sizeof(VolSet) % sizeof(unsigned) == 0, "table of whole words");
  CL_TRY(put(dvols, vols.data(), sizeof(Vol) * (size_t)n));
  CL_TRY(put(dsets, sets.data(), sizeof(VolSet) * sets.size()));
  CL_TRY(put(dpre, pre.data(), sizeof(long long) * pre.size()));
  CL_CHECK(cudaMemsetAsync(counters, 0, sizeof(int) * nctr, st));
  auto kern = batchk::k_rl_batch;
  CL_CHECK(smem_opt_in(reinterpret_cast<const void*>(kern), smem));
  int per_sm = 1, sms = 148;
#ifndef CLARITY_HOST_EMULATION
  int dev = 0;
  CL_CHECK(cudaGetDevice(&dev));
  CL_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  CL_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 256, smem));
  if (per_sm < 1) per_sm = 1;
#endif
  const long long grid = std::min<long long>(q.total, (long long)per_sm * sms);
  note_launch_begin(KK_OTHER, st);
  CLARITY_LAUNCH(kern, (unsigned)grid, 256, smem, st)(dvols, dsets, dpre, q);
  note_launch_end(KK_OTHER, st);
  CL_CHECK(cudaGetLastError());
  return Status::Ok();
}

}  // namespace clarity
