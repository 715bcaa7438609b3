// plan.hpp -- FFT plan for one padded work box (nx, ny, nz).
//
// The 3-D real transform the reference takes with FFTW/cuFFT on every call
// (src/FFT.cxx:46-146: unnormalised r2c with x halved, c2r back) is split
// into two fused passes over HBM:
//
//   XY pass  one thread block per (z, group of G consecutive y0):
//            x r2c of the G*Ay rows y = y0 + By*j (j < Ay) in shared memory,
//            then the length-Ay DFT over j and the twiddle w_ny^(y0*k1)
//            (four-step split of the y axis, ny = Ay*By).
//   Z pass   one thread block per (k1, group of W x-frequencies): the
//            length-By DFT over y0 and the full z DFT, the spectral
//            operation (OTF multiply, Wiener filter, ...), then the inverse
//            z and By transforms, all in shared memory.
//
// Spectrum layout in HBM ("S layout", complex float):
//   S[k1][kg][z][y0][ki]   k1 < Ay, kg < KG, z < nz, y0 < By, ki < W,
//   with x-frequency kx = kg*W + ki (natural order, kx < XS <= KG*W).
// A Z-pass tile S[k1][kg] is one contiguous block of nz*By*W elements.  The
// order of the y0 and z frequencies inside a tile is the digit-reversed
// order the in-place register passes leave; it never leaves the library and
// the OTF is produced by the same passes, so products line up.
#pragma once
#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

namespace clarity {

constexpr int kMaxPasses = 4;

// One complex DFT length n as register passes in decimation-in-frequency
// order.  Pass s works on sub-transforms of length len[s]; a register line
// of pass s holds radix[s] elements spaced span[s] = len[s]/radix[s] apart.
struct AxisPlan {
  int n;
  int npass;
  int radix[kMaxPasses];
  int len[kMaxPasses];
  int span[kMaxPasses];
  int tw_off;  // offset of the w_n^t (t < n) table in the twiddle buffer
};

struct VolPlan {
  int nx, ny, nz;
  int xmode;   // 0: nx even (half-length complex + r2c split); 1: nx odd
  int M;       // complex row length in the XY pass (nx/2 or nx)
  int XS;      // x-frequency slots (M+1 or nx)
  int items;   // r2c work items per row group (pairs k, M-k)
  int Ay, By;  // ny = Ay * By
  int G;       // y0 values per XY tile (divides By)
  int W;       // x-frequency slots per Z tile
  int KG;      // ceil(XS / W)
  int rowStride;  // float2 per row in XY shared memory (padded)
  int padShift;   // XY smem index p -> p + (p >> padShift)
  AxisPlan ax;    // length M
  AxisPlan ayB;   // length By
  AxisPlan az;    // length nz
  int tw_r2c_off;   // w_nx^k, k <= M/2          (even mode)
  int tw_ny_off;    // w_ny^t, t < ny            (y split twiddle)
  int xrev_off;     // int table: natural k -> smem slot after x passes
  int twiddle_count;  // float2 entries in the twiddle buffer
  int xrev_count;
  long long spec_elems;  // Ay*KG*nz*By*W
  int xy_blocks, z_blocks;
  int xy_threads, z_threads;
  int xy_smem, z_smem;   // bytes of dynamic shared memory
  long long n_real() const { return (long long)nx * ny * nz; }
};

#if defined(__CUDACC__) && !defined(CLARITY_HOST_EMULATION)
#define CLARITY_HD __host__ __device__
#else
#define CLARITY_HD
#endif

// Twiddle table w_n^t = exp(-2 pi i t / n), t < count, at float2 offset off.
struct TwTable {
  int off, n, count;
};
constexpr int kPlanTwTables = 5;

// The smem slot of natural x frequency k after the x DIF passes (digits of
// k in the passes' radices, each times its pass's span).
CLARITY_HD inline int xrev_slot(const AxisPlan& ax, int k) {
  int rem = k, pos = 0;
  for (int s = 0; s < ax.npass; ++s) {
    const int d = rem % ax.radix[s];
    rem /= ax.radix[s];
    pos += d * ax.span[s];
  }
  return pos;
}

// The twiddle tables a plan needs (x, y0 and z passes, the r2c split, the y
// split), kPlanTwTables of them; fills `out` without allocating.
inline void plan_twiddle_tables(const VolPlan& P, TwTable out[kPlanTwTables]) {
  const int m = P.M > 1 ? P.M : 1, by = P.By > 1 ? P.By : 1, nz = P.nz > 1 ? P.nz : 1;
  out[0] = TwTable{P.ax.tw_off, m, m};
  out[1] = TwTable{P.ayB.tw_off, by, by};
  out[2] = TwTable{P.az.tw_off, nz, nz};
  out[3] = TwTable{P.tw_r2c_off, P.nx, P.M / 2 + 1};
  out[4] = TwTable{P.tw_ny_off, P.ny, P.ny};
}

// The digit-reversed slot of each natural x frequency (xrev_slot), and the
// twiddle tables (plan_twiddle_tables), as vectors.
void plan_tables(const VolPlan& P, std::vector<int>* xrev, std::vector<TwTable>* tabs);

// Planner (host only).  Returns false for shapes it cannot decompose.
bool make_plan(int nx, int ny, int nz, VolPlan* out, std::string* why);
// Up to max_out (<= 8) tilings of the box, best model score first (the first
// is make_plan's); the autotuner times them.  Returns how many.
int make_plan_candidates(int nx, int ny, int nz, VolPlan* out, int max_out, std::string* why);

// Kernel families of the launch accounting and timing probes.
enum KernelKind { KK_XY_FORWARD = 0, KK_Z = 1, KK_XY_INV_FWD = 2, KK_XY_INVERSE = 3,
                  KK_OTHER = 4, KK_XY_PRODUCT = 5, KK_COUNT = 6 };

// Timing family of a launch: the functor's own kFamily when it names one
// (the RL product step, whose xy inverse+forward launches are timed apart
// from the ratio step's), else the pass's default.
template <class F, int DEF>
constexpr int family_of() {
  if constexpr (requires { F::kFamily; }) return F::kFamily;
  else return DEF;
}

// Radices accepted for one register pass (must match dft_codelets.cuh).
constexpr int kRadixSet[] = {16, 19, 17, 13, 12, 11, 10, 9, 8, 7, 6, 5, 4, 3, 2};

}  // namespace clarity
