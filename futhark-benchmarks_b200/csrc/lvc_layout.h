// Host/device shared layout definitions for the LocVolCalib engine.
//
// A *calibration* is one call of the reference entry point
// (finpar/LocVolCalib.fut:238-252): scalars outer, numX, numY, numT, s0, t,
// alpha, nu, beta.  An *instance* is one strike of one calibration (one call
// of `value`, :211-236).  Everything that does not depend on the strike --
// the grids, the operator stencils, the per-step timeline and the
// tridiagonal pivots of every time step -- is built once per calibration by
// the setup and pivot kernels into an operator-table arena in HBM; the
// rollback kernel then advances each instance's grid on chip.
#pragma once
#include <stdint.h>

#ifdef __CUDACC__
#define LVC_HD __host__ __device__ __forceinline__
#else
#define LVC_HD inline
#endif

namespace lvc {

constexpr int kKY = 16;          // rows per Y-sweep unit (one warp, 32 columns)
constexpr int kMaxCluster = 16;  // CTAs per instance (16 needs the non-portable opt-in)

// One calibration, as the device sees it.  Filled by the host runtime.
struct CalibDev {
  int32_t numX, numY, numT, Xp;    // Xp: numX padded to a power of two >= 8
  int32_t outer, xindex, yindex, C;  // C: CTAs (cluster size) per instance
  double s0, t, alpha, nu, beta;
  int64_t tab;  // offset (doubles) of the operator tables in the table arena
  int64_t piv;  // offset (elements) of the X-direction pivots in the pivot arena
  int64_t out;  // index of this calibration's first price in the output vector
};

LVC_HD int64_t al2(int64_t n) { return (n + 1) & ~int64_t(1); }

// Operator-table layout, offsets in doubles from CalibDev::tab.  Every
// sub-table starts on a 16-byte boundary.
struct TabLayout {
  int64_t colc;   // [Xp][4]  eX_i = exp(2*beta*log x_i), 0.5*Dxx_i[0..2]   (zero for i >= numX)
  int64_t rowc;   // [Y][4]   0.5*nu^2*Dyy_j[0..2], 0
  int64_t x;      // [Xp]     the spot grid myX (zero padded)
  int64_t dtinv;  // [T-1]    1/(t_{k+1} - t_k)
  int64_t eyt;    // [T-1][eyt_ld]  exp(2*(y_j - 0.5*nu^2*t_k))
  int64_t yco;    // [T-1][Y][4]    Y-sweep multipliers: mY_j, nY_j, 1/b'_j, 0
  int64_t total;
  int64_t eyt_ld;
};

LVC_HD TabLayout tab_layout(int X, int Y, int T, int Xp) {
  (void)X;
  TabLayout L;
  const int64_t steps = T > 1 ? T - 1 : 0;
  L.colc = 0;
  L.rowc = L.colc + 4LL * Xp;
  L.x = L.rowc + 4LL * Y;
  L.dtinv = L.x + Xp;
  L.eyt_ld = al2(Y);
  L.eyt = L.dtinv + al2(steps);
  L.yco = L.eyt + steps * L.eyt_ld;
  L.total = L.yco + steps * 4LL * Y;
  return L;
}

// Elements of the X-direction pivot array rbX[T-1][Y][Xp] of one calibration.
LVC_HD int64_t piv_elems(int Y, int T, int Xp) {
  return (T > 1 ? (int64_t)(T - 1) : 0) * Y * Xp;
}

// Row padding of the on-chip grid: PADS elements after every 8, so that the
// 16-byte vector loads of 8-element row chunks by consecutive lanes hit
// distinct shared-memory banks (80-byte chunk stride for f64, 48 for f32).
template <typename S> struct Pad;
template <> struct Pad<double> { static constexpr int v = 2; };
template <> struct Pad<float> { static constexpr int v = 4; };

template <typename S> LVC_HD int row_ld(int Xp) { return Xp + (Xp / 8) * Pad<S>::v; }
template <typename S> LVC_HD int col_off(int i) { return i + (i >> 3) * Pad<S>::v; }

LVC_HD int ceil_div(int a, int b) { return (a + b - 1) / b; }

// Shared-memory carve-up of the rollback kernel for one CTA holding `Ycs`
// rows of a grid with padded width Xp and numX real columns.  Offsets are in
// elements of S; every region is 16-byte aligned.  With onchip == false the
// two grid buffers A and B live in HBM instead and take no shared memory.
struct SmemLayout {
  int LD, Ycs, G, P, U;
  int A, B, colc, rowc, tab0, tab1, tabsz, aggF, aggB, blkF, blkB, zin, xin, misc, total;
  int grid_elems;
};

template <typename S> LVC_HD SmemLayout smem_layout(int Xp, int X, int Ycs, bool onchip) {
  const int a = 16 / (int)sizeof(S);  // elements per 16 bytes
  auto up = [a](int n) { return (n + a - 1) / a * a; };
  SmemLayout L;
  L.LD = row_ld<S>(Xp);
  L.Ycs = Ycs;
  L.G = ceil_div(X, 32);
  L.P = ceil_div(Ycs, kKY);
  L.U = L.G * L.P;
  int o = 0;
  L.A = o; if (onchip) o += up(Ycs * L.LD);
  L.B = o; if (onchip) o += up(Ycs * L.LD);
  L.colc = o; o += up(4 * Xp);
  L.rowc = o; o += up(4 * Ycs);
  // per-step tables: eyt, mY, nY, rbY, cp, cq  (6*Ycs) + BF, BB (2*P) + 2 block totals
  L.tabsz = up(6 * Ycs + 2 * L.P + 2);
  L.tab0 = o; o += L.tabsz;
  L.tab1 = o; o += L.tabsz;
  L.aggF = o; o += up(L.U * 32);
  L.aggB = o; o += up(L.U * 32);
  L.blkF = o; o += up(L.G * 32);
  L.blkB = o; o += up(L.G * 32);
  L.zin = o; o += up(L.G * 32);
  L.xin = o; o += up(L.G * 32);
  L.misc = o; o += up(8);
  L.total = o;
  L.grid_elems = 2 * up(Ycs * L.LD);  // A + B, wherever they live
  return L;
}

// Offsets inside one per-step table block (elements of S).
struct StepTab {
  int eyt, mY, nY, rbY, cp, cq, BF, BB, blkBF, blkBB;
};
LVC_HD StepTab step_tab(int Ycs, int P) {
  StepTab t;
  t.eyt = 0;
  t.mY = Ycs;
  t.nY = 2 * Ycs;
  t.rbY = 3 * Ycs;
  t.cp = 4 * Ycs;
  t.cq = 5 * Ycs;
  t.BF = 6 * Ycs;
  t.BB = 6 * Ycs + P;
  t.blkBF = 6 * Ycs + 2 * P;
  t.blkBB = 6 * Ycs + 2 * P + 1;
  return t;
}

// Work item of the rollback kernel: calibration index and strike index.
struct Item {
  int32_t calib, strike;
};

}  // namespace lvc
