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
constexpr int kLineK = 16;       // line-kernel chunk: elements of a line per lane

// Rollback kernel family of a calibration.
enum : int32_t {
  kKindChunk = 0,  // lanes own 8/16-element chunks of a row (any numX <= 512, HBM-state capable)
  kKindLine = 1,   // lanes own whole lines of the grid (numX <= 256, on chip)
};

// One calibration, as the device sees it.  Filled by the host runtime.
struct CalibDev {
  int32_t numX, numY, numT, Xp;      // Xp: numX padded to a power of two >= 8
  int32_t outer, xindex, yindex, C;  // C: CTAs (cluster size) per instance
  int32_t kind, Ycs, ld, pad1;       // kernel family; rows per CTA; line family: row stride
  double s0, t, alpha, nu, beta;
  int64_t tab;  // offset (doubles) of the operator tables in the table arena
  int64_t piv;  // offset (elements) of the X-direction pivots in the pivot arena
  int64_t out;  // index of this calibration's first price in the output vector
};
static_assert(sizeof(CalibDev) == 112, "bench.py counts 112 uploaded bytes per calibration");

LVC_HD int64_t al2(int64_t n) { return (n + 1) & ~int64_t(1); }

// Operator-table layout, offsets in doubles from CalibDev::tab.  Every
// sub-table starts on a 16-byte boundary.  Shared by both kernel families:
// colc, rowc, x, dtinv.  Chunk family: eyt, yco.  Line family: wcol, stab.
struct TabLayout {
  int64_t colc;   // [Xp][4]  eX_i = exp(2*beta*log x_i), 0.5*Dxx_i[0..2]   (zero for i >= numX)
  int64_t rowc;   // [Y][4]   0.5*nu^2*Dyy_j[0..2], 0
  int64_t x;      // [Xp]     the spot grid myX (zero padded)
  int64_t dtinv;  // [T-1]    1/(t_{k+1} - t_k)
  int64_t eyt;    // [T-1][eyt_ld]  exp(2*(y_j - 0.5*nu^2*t_k))            (chunk family)
  int64_t yco;    // [T-1][Y][4]    Y-sweep multipliers: mY_j, nY_j, 1/b'_j, 0  (chunk family)
  int64_t wcol;   // [3][xa]  W_k(i) = 0.25 * eX_i * Dxx_i[k]                 (line family)
  int64_t stab;   // [T-1][Y][8]    step-table rows, slots kSlot* below       (line family)
  int64_t total;
  int64_t eyt_ld, xa;
};

LVC_HD TabLayout tab_layout(int X, int Y, int T, int Xp, int kind) {
  TabLayout L;
  const int64_t steps = T > 1 ? T - 1 : 0;
  L.xa = al2(X);
  L.eyt_ld = al2(Y);
  L.colc = 0;
  L.rowc = L.colc + 4LL * Xp;
  L.x = L.rowc + 4LL * Y;
  L.dtinv = L.x + Xp;
  int64_t o = L.dtinv + al2(steps);
  if (kind == kKindChunk) {
    L.eyt = o;
    o += steps * L.eyt_ld;
    L.yco = o;
    o += steps * 4LL * Y;
    L.wcol = L.stab = o;
  } else {
    L.wcol = o;
    o += 3 * L.xa;
    L.stab = o;
    o += steps * 8LL * Y;
    L.eyt = L.yco = o;
  }
  L.total = o;
  return L;
}

// Slots of a line-family step-table row (8 doubles; slots 5 and 7 are zero).
// The pair that kernels read as one 16-byte vector, (nY, 1/b'), starts on an
// even slot.
enum : int {
  kSlotE = 0,   // exp(2 (y_j - 0.5 nu^2 t_k))
  kSlotMY = 1,  // forward multiplier -a_j / b'_{j-1}
  kSlotNY = 2,  // backward multiplier -c_j / b'_j
  kSlotRB = 3,  // 1 / b'_j
  kSlotCQ = 4,  // suffix product of nY inside the chunk
  kSlotCP = 6,  // prefix product of mY inside the chunk
};

// Line family: the pivot rows are stored exactly as the kernel's shared-memory
// image of them -- row j of step k at ((k*Y4 + j) * LD) -- so one bulk copy
// moves a CTA's rows.  The row stride is CalibDev::ld: the odd LD = numX | 1
// (8-byte accesses down a column conflict-free) for the line and full-tile
// kernels, LD = numX + 2 (2 mod 4: 16-byte pair accesses conflict-free and
// aligned) for the paired kernel.
LVC_HD int line_ld(int X) { return X | 1; }
LVC_HD int pair_ld(int X) { return X + 2; }
LVC_HD int64_t round4(int64_t n) { return (n + 3) & ~int64_t(3); }

// Elements of the X-direction pivot array of one calibration (plus 4 of
// padding so that bulk copies rounded up to 16 bytes stay in bounds):
// chunk family rbX[T-1][Y][Xp]; line family rbL[T-1][Y4][ld].
LVC_HD int64_t piv_elems(int X, int Y, int T, int Xp, int kind, int ld) {
  const int64_t steps = T > 1 ? (int64_t)(T - 1) : 0;
  return kind == kKindChunk ? steps * Y * Xp : steps * round4(Y) * ld + 4;
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
  int grid_elems;            // per-CTA HBM scratch when !onchip: A, B, aggF, aggB
  int gA, gB, gaggF, gaggB;  // their offsets in that scratch
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
  L.aggF = o; if (onchip) o += up(L.U * 32);
  L.aggB = o; if (onchip) o += up(L.U * 32);
  L.blkF = o; o += up(L.G * 32);
  L.blkB = o; o += up(L.G * 32);
  L.zin = o; o += up(L.G * 32);
  L.xin = o; o += up(L.G * 32);
  L.misc = o; o += up(8);
  L.total = o;
  L.gA = 0;
  L.gB = up(Ycs * L.LD);
  L.gaggF = 2 * up(Ycs * L.LD);
  L.gaggB = L.gaggF + up(L.U * 32);
  L.grid_elems = onchip ? 2 * up(Ycs * L.LD) : L.gaggB + up(L.U * 32);
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
