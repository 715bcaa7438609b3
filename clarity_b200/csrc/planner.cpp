// planner.cpp -- host-only planning of the fused FFT passes for one work
// box (see plan.hpp for the pass structure and the S layout).
#include <algorithm>
#include <climits>
#include <cstring>
#include <string>
#include <vector>

#include "plan.hpp"

namespace clarity {

static void search_axis(int n, int depth, int* cur, int* best, int* best_len,
                        int* best_max) {
  if (n == 1) {
    int mx = 0;
    for (int i = 0; i < depth; ++i) mx = std::max(mx, cur[i]);
    if (depth < *best_len || (depth == *best_len && mx < *best_max)) {
      *best_len = depth;
      *best_max = mx;
      for (int i = 0; i < depth; ++i) best[i] = cur[i];
    }
    return;
  }
  if (depth >= kMaxPasses || depth + 1 > *best_len) return;
  for (int r : kRadixSet) {
    if (n % r == 0) {
      // keep radices non-increasing to avoid permutations of one factor set
      if (depth > 0 && r > cur[depth - 1]) continue;
      cur[depth] = r;
      search_axis(n / r, depth + 1, cur, best, best_len, best_max);
    }
  }
}

static bool plan_axis(int n, AxisPlan* A) {
  std::memset(A, 0, sizeof(*A));
  A->n = n;
  if (n == 1) return true;
  int cur[kMaxPasses], best[kMaxPasses];
  int best_len = kMaxPasses + 1, best_max = INT_MAX;
  search_axis(n, 0, cur, best, &best_len, &best_max);
  if (best_len > kMaxPasses) return false;
  A->npass = best_len;
  int len = n;
  for (int s = 0; s < best_len; ++s) {
    A->radix[s] = best[s];
    A->len[s] = len;
    A->span[s] = len / best[s];
    len /= best[s];
  }
  return true;
}

static int ctz(int v) {
  int c = 0;
  while (v && !(v & 1)) { v >>= 1; ++c; }
  return c;
}

static constexpr int kSmemMax = 200 * 1024;
static constexpr int kSmemPerSM = 228 * 1024;

// Fills the offsets of a chosen tiling (spectrum size, twiddle layout);
// false when 32-bit offsets would not address the box.
static bool finalize_plan(VolPlan& P, std::string* why) {
  const long long spec = (long long)P.Ay * P.KG * P.nz * P.By * P.W;
  if ((long long)P.nx * P.ny * P.nz >= (1ll << 31) || spec >= (1ll << 31)) {
    if (why) *why = "work box of 2^31 voxels or more";
    return false;
  }
  P.xy_threads = 256;
  P.z_threads = 256;
  P.spec_elems = spec;
  int off = 0;
  P.ax.tw_off = off; off += std::max(P.M, 1);
  P.ayB.tw_off = off; off += std::max(P.By, 1);
  P.az.tw_off = off; off += std::max(P.nz, 1);
  P.tw_r2c_off = off; off += P.M / 2 + 1;
  P.tw_ny_off = off; off += P.ny;
  P.twiddle_count = off;
  P.xrev_off = 0;
  P.xrev_count = P.M;
  return true;
}

bool make_plan(int nx, int ny, int nz, VolPlan* out, std::string* why) {
  return make_plan_candidates(nx, ny, nz, out, 1, why) > 0;
}

int make_plan_candidates(int nx, int ny, int nz, VolPlan* out, int max_out, std::string* why) {
  VolPlan P;
  std::memset(&P, 0, sizeof(P));
  P.nx = nx; P.ny = ny; P.nz = nz;
  P.xmode = (nx % 2 == 0) ? 0 : 1;
  P.M = P.xmode == 0 ? nx / 2 : nx;
  P.XS = P.xmode == 0 ? P.M + 1 : nx;
  if (P.xmode == 0)
    P.items = (P.M % 2 == 0) ? std::max(P.M / 2, 1) : (P.M + 1) / 2;
  else
    P.items = nx;
  if (!plan_axis(P.M, &P.ax)) {
    if (why) *why = "x length " + std::to_string(nx) + " has an unsupported factor";
    return false;
  }
  if (!plan_axis(nz, &P.az)) {
    if (why) *why = "z length " + std::to_string(nz) + " has an unsupported factor";
    return false;
  }
  // x row padding in the XY shared memory
  if (P.ax.npass <= 1 || (P.ax.span[0] & 1)) P.padShift = 30;
  else P.padShift = ctz(P.ax.span[0]);
  {
    const int last = P.M - 1;
    int rs = last + (last >> P.padShift) + 1;
    if (rs % 2 == 0) rs += 1;
    P.rowStride = rs;
  }
  // the max_out best-scoring tilings, best first (insertion into a fixed
  // array: planning allocates nothing)
  constexpr int kMaxCand = 8;
  if (max_out > kMaxCand) max_out = kMaxCand;
  if (max_out < 1) max_out = 1;
  VolPlan cand[kMaxCand];
  double cscore[kMaxCand];
  int ncand = 0;
  // candidate Ay: 1 and every register radix (fixed array: planning
  // allocates nothing)
  int ays[1 + sizeof(kRadixSet) / sizeof(kRadixSet[0])];
  int nays = 0;
  ays[nays++] = 1;
  for (int r : kRadixSet) ays[nays++] = r;
  for (int ai = 0; ai < nays; ++ai) {
    const int ay = ays[ai];
    if (ny % ay) continue;
    const int by = ny / ay;
    AxisPlan ab;
    if (!plan_axis(by, &ab)) continue;
    for (int W : {1, 2, 4, 8}) {
      const long long zsm = (long long)nz * by * W * 8;
      if (zsm > kSmemMax) continue;
      for (int G = 1; G <= 16; ++G) {
        if (by % G) continue;
        const long long xysm = (long long)G * ay * P.rowStride * 8;
        if (xysm > kSmemMax) continue;
        const int KG = (P.XS + W - 1) / W;
        const long long xy_blocks = (long long)nz * (by / G);
        const long long z_blocks = (long long)ay * KG;
        const int occ_xy = std::min(8, (int)(kSmemPerSM / (xysm + 1024)));
        const int occ_z = std::min(8, (int)(kSmemPerSM / (zsm + 1024)));
        const double seg = (double)G * W * 8;
        double score = 0;
        score += 10.0 * std::min(std::min(occ_xy, occ_z), 3);
        score += seg >= 32 ? 6.0 : seg / 32.0 * 6.0;
        score += (xy_blocks >= 296 ? 3.0 : 3.0 * xy_blocks / 296.0);
        score += (z_blocks >= 296 ? 3.0 : 3.0 * z_blocks / 296.0);
        score -= 4.0 * ((double)KG * W / P.XS - 1.0);
        score -= 0.05 * std::abs(ay - 16);
        score -= 0.02 * G;  // prefer fewer rows per tile at equal merit
        int pos = ncand;
        while (pos > 0 && score > cscore[pos - 1]) --pos;
        if (pos < max_out) {
          const int last = std::min(ncand, max_out - 1);
          for (int q = last; q > pos; --q) {
            cand[q] = cand[q - 1];
            cscore[q] = cscore[q - 1];
          }
          VolPlan c = P;
          c.Ay = ay; c.By = by; c.G = G; c.W = W; c.KG = KG;
          c.ayB = ab;
          c.xy_smem = (int)xysm;
          c.z_smem = (int)zsm;
          c.xy_blocks = (int)xy_blocks;
          c.z_blocks = (int)z_blocks;
          cand[pos] = c;
          cscore[pos] = score;
          if (ncand < max_out) ++ncand;
        }
      }
    }
  }
  if (ncand == 0) {
    if (why) *why = "no tiling of y=" + std::to_string(ny) + ", z=" + std::to_string(nz) +
                    " fits in shared memory with the supported radices";
    return 0;
  }
  int nout = 0;
  for (int c = 0; c < ncand; ++c)
    if (finalize_plan(cand[c], why)) out[nout++] = cand[c];
  return nout;
}


void plan_tables(const VolPlan& P, std::vector<int>* xrev, std::vector<TwTable>* tabs) {
  xrev->assign(std::max(P.M, 1), 0);
  for (int k = 0; k < P.M; ++k) (*xrev)[k] = xrev_slot(P.ax, k);
  TwTable t[kPlanTwTables];
  plan_twiddle_tables(P, t);
  tabs->assign(t, t + kPlanTwTables);
}

}  // namespace clarity
