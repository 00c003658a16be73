// Device kernels of the LocVolCalib engine (sm_100a).
//
//   lvc_setup_kernel    initGrid + initOperator + the strike-independent
//                       per-step tables (finpar/LocVolCalib.fut:12-44, :50-66)
//                       and the Y-direction LU pivots of every step.
//   lvc_pivot_kernel    the X-direction LU pivots 1/b'_i of every (step, row)
//                       (recurrence 1 of tridagPar, :71-91), strike-independent.
//   lvc_rollback_kernel persistent: one CTA (or a thread-block cluster) per
//                       strike instance, the whole numY x numX grid resident in
//                       shared memory for all numT-1 steps; each step is
//                       explicitX + explicitY + implicitX + implicitY
//                       (:180-209) with the two linear recurrences of tridagPar
//                       (:96-123) solved as chunked warp/CTA/cluster scans.
#pragma once
#include <cooperative_groups.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "lvc_layout.h"

namespace lvc {
namespace cg = cooperative_groups;

// ---------------------------------------------------------------------------
// setup kernel: one CTA per calibration.  The grid and stencil formulas use
// explicitly rounded operations (no FMA contraction) so the tables are the
// reference's IEEE f64 values.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double grid_pt(int i, double d, double idx, double base) {
  // f32.i64 i * d - f32.i32 index * d + base   (:21-22)
  return __dadd_rn(__dsub_rn(__dmul_rn((double)i, d), __dmul_rn(idx, d)), base);
}

// Second-derivative stencil DD of initOperator (:26-44) at interior point i.
__device__ __forceinline__ void dd_stencil(double xm, double x0, double xp, double& d0,
                                           double& d1, double& d2) {
  const double dxl = __dsub_rn(x0, xm);
  const double dxu = __dsub_rn(xp, x0);
  const double s = __dadd_rn(dxl, dxu);
  d0 = __ddiv_rn(__ddiv_rn(2.0, dxl), s);
  d1 = __ddiv_rn(__dmul_rn(-2.0, __dadd_rn(__ddiv_rn(1.0, dxl), __ddiv_rn(1.0, dxu))), s);
  d2 = __ddiv_rn(__ddiv_rn(2.0, dxu), s);
}

__global__ void __launch_bounds__(256) lvc_setup_kernel(const CalibDev* __restrict__ calibs,
                                                        double* __restrict__ tabs) {
  const CalibDev c = calibs[blockIdx.x];
  const int X = c.numX, Y = c.numY, T = c.numT, Xp = c.Xp;
  const bool line = c.kind == kKindLine;
  const TabLayout L = tab_layout(X, Y, T, Xp, c.kind);
  double* tab = tabs + c.tab;
  const int tid = threadIdx.x, nt = blockDim.x;

  // initGrid (:12-23)
  const double logAlpha = log(c.alpha);
  const double sqt = sqrt(c.t);
  const double stdX = __dmul_rn(__dmul_rn(__dmul_rn(20.0, c.alpha), c.s0), sqt);
  const double stdY = __dmul_rn(__dmul_rn(10.0, c.nu), sqt);
  const double dx = __ddiv_rn(stdX, (double)X);
  const double dy = __ddiv_rn(stdY, (double)Y);
  const double xidx = (double)c.xindex, yidx = (double)c.yindex;
  const double half_nu2 = __dmul_rn(0.5, __dmul_rn(c.nu, c.nu));  // 0.5 * var, var = nu*nu
  const double half_nu_nu = __dmul_rn(__dmul_rn(0.5, c.nu), c.nu);  // 0.5 * nu * nu

  // Column tables: eX_i and 0.5 * Dxx_i[k]  (updateParams :63, explicitMethod :138-144)
  for (int i = tid; i < Xp; i += nt) {
    double e = 0.0, h0 = 0.0, h1 = 0.0, h2 = 0.0, xv = 0.0;
    if (i < X) {
      xv = grid_pt(i, dx, xidx, c.s0);
      e = exp(__dmul_rn(2.0, __dmul_rn(c.beta, log(xv))));
      if (i > 0 && i < X - 1) {
        double d0, d1, d2;
        dd_stencil(grid_pt(i - 1, dx, xidx, c.s0), xv, grid_pt(i + 1, dx, xidx, c.s0), d0, d1,
                   d2);
        h0 = __dmul_rn(0.5, d0);
        h1 = __dmul_rn(0.5, d1);
        h2 = __dmul_rn(0.5, d2);
      }
    }
    double* cc = tab + L.colc + 4LL * i;
    cc[0] = e;
    cc[1] = h0;
    cc[2] = h1;
    cc[3] = h2;
    tab[L.x + i] = xv;
    // line family: W_k = 0.25 * eX_i * Dxx_i[k], so that 0.5 * (0.5 * VarX * Dxx[k]) = e_j * W_k
    if (line && i < L.xa) {
      tab[L.wcol + i] = 0.5 * (e * h0);
      tab[L.wcol + L.xa + i] = 0.5 * (e * h1);
      tab[L.wcol + 2 * L.xa + i] = 0.5 * (e * h2);
    }
  }
  // Row tables: 0.5 * nu^2 * Dyy_j[k]
  for (int j = tid; j < Y; j += nt) {
    double g0 = 0.0, g1 = 0.0, g2 = 0.0;
    if (j > 0 && j < Y - 1) {
      double d0, d1, d2;
      dd_stencil(grid_pt(j - 1, dy, yidx, logAlpha), grid_pt(j, dy, yidx, logAlpha),
                 grid_pt(j + 1, dy, yidx, logAlpha), d0, d1, d2);
      g0 = __dmul_rn(half_nu2, d0);
      g1 = __dmul_rn(half_nu2, d1);
      g2 = __dmul_rn(half_nu2, d2);
    }
    double* rc = tab + L.rowc + 4LL * j;
    rc[0] = g0;
    rc[1] = g1;
    rc[2] = g2;
    rc[3] = 0.0;
  }
  const int steps = T > 1 ? T - 1 : 0;
  const double tden = __dsub_rn((double)T, 1.0);
  // timeline t_k = t * k / (numT - 1) (:14), dtInv (:193), exp(2(y_j - 0.5 nu^2 t_k))
  for (int k = tid; k < steps; k += nt) {
    const double tn = __ddiv_rn(__dmul_rn(c.t, (double)k), tden);
    const double tx = __ddiv_rn(__dmul_rn(c.t, (double)(k + 1)), tden);
    tab[L.dtinv + k] = __ddiv_rn(1.0, __dsub_rn(tx, tn));
  }
  for (int64_t e = tid; e < (int64_t)steps * Y; e += nt) {
    const int k = (int)(e / Y), j = (int)(e % Y);
    const double tn = __ddiv_rn(__dmul_rn(c.t, (double)k), tden);
    const double yj = grid_pt(j, dy, yidx, logAlpha);
    const double ev = exp(__dmul_rn(2.0, __dsub_rn(yj, __dmul_rn(half_nu_nu, tn))));
    if (line)
      tab[L.stab + ((int64_t)k * Y + j) * 8] = ev;
    else
      tab[L.eyt + (int64_t)k * L.eyt_ld + j] = ev;
  }
  __syncthreads();  // row tables and dtInv are visible to the whole CTA

  // Y-direction pivots of every step (implicitY: one matrix per step, shared
  // by every column and every strike): b'_j = b_j - a_j c_{j-1} / b'_{j-1}.
  for (int k = tid; k < steps; k += nt) {
    const double dt = tab[L.dtinv + k];
    double rb_prev = 0.0, c_prev = 0.0;
    double* yc = line ? tab + L.stab + 8LL * k * Y : tab + L.yco + 4LL * k * Y;
    const int w = line ? 8 : 4, o = line ? 1 : 0;
    for (int j = 0; j < Y; j++) {
      const double* rc = tab + L.rowc + 4LL * j;
      const double a = -(0.5 * rc[0]);
      const double b = dt - 0.5 * rc[1];
      const double cc = -(0.5 * rc[2]);
      const double bp = (j == 0) ? b : b - a * c_prev * rb_prev;
      const double rb = 1.0 / bp;
      yc[w * j + o + 0] = (j == 0) ? 0.0 : -a * rb_prev;  // forward multiplier -a_j / b'_{j-1}
      yc[w * j + o + 1] = (j == Y - 1) ? 0.0 : -cc * rb;  // backward multiplier -c_j / b'_j
      yc[w * j + o + 2] = rb;
      if (!line) yc[w * j + 3] = 0.0;
      rb_prev = rb;
      c_prev = cc;
    }
    if (line) {
      // products of the multipliers inside each kLineK-row chunk of each
      // CTA's row block: cp_j = prod_{chunk start..j} mY, cq_j = prod_{j..chunk end} nY
      for (int r0 = 0; r0 < Y; r0 += c.Ycs) {
        const int r1 = min(Y, r0 + c.Ycs);
        for (int jb = r0; jb < r1; jb += kLineK) {
          const int je = min(r1, jb + kLineK);
          double pr = 1.0;
          for (int j = jb; j < je; j++) {
            pr = pr * yc[8 * j + kSlotMY];
            yc[8 * j + kSlotCP] = pr;
          }
          pr = 1.0;
          for (int j = je - 1; j >= jb; j--) {
            pr = pr * yc[8 * j + kSlotNY];
            yc[8 * j + kSlotCQ] = pr;
          }
          for (int j = jb; j < je; j++) {
            yc[8 * j + 5] = 0.0;
            yc[8 * j + 7] = 0.0;
          }
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// pivot kernel: one lane per (calibration, step, row) runs the sequential pivot
// recurrence of one X-direction system, written as 1/b'_i.  A warp owns 32
// consecutive rows and goes through them 32 columns at a time: every lane
// puts its 32 pivots in a shared tile, then the warp writes the tile out one
// row at a time, 32 consecutive columns per store, so every row leaves in
// whole 32-byte sectors (a store per lane per column would touch 32 rows per
// instruction and leave partly written sectors to the L2).
// ---------------------------------------------------------------------------
constexpr int kPivotWarps = 4;  // warps per CTA (128 threads)

template <typename PV>
__global__ void __launch_bounds__(128) lvc_pivot_kernel(const CalibDev* __restrict__ calibs,
                                                        const int64_t* __restrict__ row_start,
                                                        int ncal, const double* __restrict__ tabs,
                                                        PV* __restrict__ piv) {
  __shared__ double tile[kPivotWarps][32][33];
  __shared__ PV* rowp[kPivotWarps][32];
  __shared__ int rowx[kPivotWarps][32], rowld[kPivotWarps][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t total = row_start[ncal];
  const int64_t ngroups = (total + 31) / 32;
  for (int64_t g = (int64_t)blockIdx.x * kPivotWarps + w; g < ngroups; g += (int64_t)gridDim.x * kPivotWarps) {
    const int64_t r = g * 32 + lane;
    int X = 0, LDr = 0;
    PV* o = nullptr;
    bool line = false;
    double e = 0.0, dt = 0.0;
    const double* tab = tabs;
    TabLayout L{};
    if (r < total) {
      int lo = 0, hi = ncal - 1;  // last c with row_start[c] <= r
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (row_start[mid] <= r) lo = mid; else hi = mid - 1;
      }
      const CalibDev c = calibs[lo];
      const int Y = c.numY;
      X = c.numX;
      L = tab_layout(X, Y, c.numT, c.Xp, c.kind);
      const int64_t local = r - row_start[lo];
      const int k = (int)(local / Y), j = (int)(local % Y);
      tab = tabs + c.tab;
      dt = tab[L.dtinv + k];
      line = c.kind == kKindLine;
      if (line) {
        // rows of stride ld: the line kernels' shared-memory image
        e = tab[L.stab + ((int64_t)k * Y + j) * 8];
        LDr = c.ld;
        o = piv + c.piv + ((int64_t)k * round4(Y) + j) * LDr;
      } else {
        e = tab[L.eyt + (int64_t)k * L.eyt_ld + j];
        LDr = c.Xp;
        o = piv + c.piv + ((int64_t)k * Y + j) * LDr;
      }
    }
    rowp[w][lane] = o;
    rowx[w][lane] = X;
    rowld[w][lane] = LDr;
    const int maxld = __reduce_max_sync(0xffffffffu, (unsigned)LDr);
    __syncwarp();
    double rb_prev = 0.0, c_prev = 0.0;
    for (int c0 = 0; c0 < maxld; c0 += 32) {
      for (int m = 0; m < 32; m++) {
        const int i = c0 + m;
        double rb = 0.0;
        if (i < X) {
          double a, b, cc;
          if (line) {
            // b'_i = (dt - e W1_i) - (e W0_i)(e W2_{i-1}) / b'_{i-1}
            const double* W0 = tab + L.wcol;
            a = -(e * W0[i]);
            b = dt - e * W0[L.xa + i];
            cc = -(e * W0[2 * L.xa + i]);
          } else {
            const double2 c01 = *reinterpret_cast<const double2*>(tab + L.colc + 4LL * i);
            const double2 c23 = *reinterpret_cast<const double2*>(tab + L.colc + 4LL * i + 2);
            const double var = c01.x * e;
            a = -(0.5 * (var * c01.y));
            b = dt - 0.5 * (var * c23.x);
            cc = -(0.5 * (var * c23.y));
          }
          const double bp = (i == 0) ? b : b - a * c_prev * rb_prev;
          rb = 1.0 / bp;
          rb_prev = rb;
          c_prev = cc;
        }
        tile[w][lane][m] = rb;
      }
      __syncwarp();
      for (int rr = 0; rr < 32; rr++) {
        PV* orow = rowp[w][rr];
        const int i = c0 + lane;
        if (orow && i < rowld[w][rr]) orow[i] = (PV)(i < rowx[w][rr] ? tile[w][rr][lane] : 0.0);
      }
      __syncwarp();
    }
  }
}

// ---------------------------------------------------------------------------
// rollback kernel
// ---------------------------------------------------------------------------
template <typename S, typename PV>
struct RollbackArgs {
  const CalibDev* calibs;
  const Item* items;
  int n_items;
  int C;               // CTAs per instance (== launch cluster size)
  int smem_elems;      // dynamic shared memory provided, in elements of S
  const double* tabs;  // operator-table arena
  const PV* piv;       // X-pivot arena
  double* out;         // prices
  S* gstate;           // grid state in HBM for grids too large for the chip (or null)
  int64_t gstate_per_cta;
  int* err;
};

template <typename S> struct Vec2;
template <> struct Vec2<double> { using T = double2; };
template <> struct Vec2<float> { using T = float4; };

// Load KX consecutive elements starting at column i0 (i0 % 8 == 0) of a
// padded row, as 16-byte vectors.  `row` may be a shared, distributed-shared
// (cluster peer) or global generic pointer.
template <int KX>
__device__ __forceinline__ void load_chunk(const double* row, int i0, double (&v)[KX], bool ok) {
#pragma unroll
  for (int m = 0; m < KX; m += 2) {
    double2 t = make_double2(0.0, 0.0);
    if (ok) t = *reinterpret_cast<const double2*>(row + col_off<double>(i0 + m));
    v[m] = t.x;
    v[m + 1] = t.y;
  }
}
template <int KX>
__device__ __forceinline__ void load_chunk(const float* row, int i0, float (&v)[KX], bool ok) {
#pragma unroll
  for (int m = 0; m < KX; m += 4) {
    float4 t = make_float4(0.f, 0.f, 0.f, 0.f);
    if (ok) t = *reinterpret_cast<const float4*>(row + col_off<float>(i0 + m));
    v[m] = t.x;
    v[m + 1] = t.y;
    v[m + 2] = t.z;
    v[m + 3] = t.w;
  }
}
template <int KX>
__device__ __forceinline__ void store_chunk(double* row, int i0, const double (&v)[KX]) {
#pragma unroll
  for (int m = 0; m < KX; m += 2)
    *reinterpret_cast<double2*>(row + col_off<double>(i0 + m)) = make_double2(v[m], v[m + 1]);
}
template <int KX>
__device__ __forceinline__ void store_chunk(float* row, int i0, const float (&v)[KX]) {
#pragma unroll
  for (int m = 0; m < KX; m += 4)
    *reinterpret_cast<float4*>(row + col_off<float>(i0 + m)) =
        make_float4(v[m], v[m + 1], v[m + 2], v[m + 3]);
}
// Pivot chunk from HBM/L2 (read-only path).
template <int KX>
__device__ __forceinline__ void load_piv(const double* p, double (&v)[KX], bool ok) {
#pragma unroll
  for (int m = 0; m < KX; m += 2) {
    double2 t = make_double2(0.0, 0.0);
    if (ok) t = __ldg(reinterpret_cast<const double2*>(p + m));
    v[m] = t.x;
    v[m + 1] = t.y;
  }
}
template <int KX>
__device__ __forceinline__ void load_piv(const float* p, float (&v)[KX], bool ok) {
#pragma unroll
  for (int m = 0; m < KX; m += 4) {
    float4 t = make_float4(0.f, 0.f, 0.f, 0.f);
    if (ok) t = __ldg(reinterpret_cast<const float4*>(p + m));
    v[m] = t.x;
    v[m + 1] = t.y;
    v[m + 2] = t.z;
    v[m + 3] = t.w;
  }
}

// Register budget: 128 per thread for the 8-wide chunks (several CTAs of a
// small grid may share an SM); the 16-wide chunks of numX > 256 get 255.
template <int NT, int KX> struct MinBlocks {
  static constexpr int v = KX == 16 ? 1 : (512 / NT);
};

template <typename S, typename PV, int NT, int KX, bool GSTATE>
__global__ void __launch_bounds__(NT, (MinBlocks<NT, KX>::v)) lvc_rollback_kernel(RollbackArgs<S, PV> args) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  S* sm = reinterpret_cast<S*>(smem_raw);
  constexpr int NW = NT / 32;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int C = args.C;
  const bool clustered = C > 1;
  int rank = 0;
  if (clustered) rank = (int)cg::this_cluster().block_rank();
  const int cid = blockIdx.x / C, ncl = gridDim.x / C;
  unsigned sc = 0;  // running step counter: selects the double-buffered step tables

  for (int it = cid; it < args.n_items; it += ncl) {
    const Item item = args.items[it];
    const CalibDev c = args.calibs[item.calib];
    const int X = c.numX, Y = c.numY, T = c.numT, Xp = c.Xp;
    const int Ycs = ceil_div(Y, C);
    const int r0 = rank * Ycs;
    const int Yc = max(0, min(Ycs, Y - r0));
    const SmemLayout Lf = smem_layout<S>(Xp, X, Ycs, !GSTATE);
    // Uniform over the cluster: every CTA of a cluster sees the same item.
    if (c.C != C || Xp / KX > 32 || Xp % KX != 0 || Lf.total > args.smem_elems ||
        (GSTATE && Lf.grid_elems > args.gstate_per_cta)) {
      if (tid == 0) atomicExch(args.err, 1);
      continue;
    }
    const int LD = Lf.LD;
    S* A;
    S* B;
    S* s_aggF;
    S* s_aggB;
    if constexpr (GSTATE) {
      S* g = args.gstate + (int64_t)blockIdx.x * args.gstate_per_cta;
      A = g + Lf.gA;
      B = g + Lf.gB;
      s_aggF = g + Lf.gaggF;
      s_aggB = g + Lf.gaggB;
    } else {
      A = sm + Lf.A;
      B = sm + Lf.B;
      s_aggF = sm + Lf.aggF;
      s_aggB = sm + Lf.aggB;
    }
    S* s_colc = sm + Lf.colc;
    S* s_rowc = sm + Lf.rowc;
    S* s_tab[2] = {sm + Lf.tab0, sm + Lf.tab1};
    S* s_blkF = sm + Lf.blkF;
    S* s_blkB = sm + Lf.blkB;
    S* s_zin = sm + Lf.zin;
    S* s_xin = sm + Lf.xin;
    const StepTab st = step_tab(Ycs, Lf.P);
    const double* tabc = args.tabs + c.tab;
    const TabLayout Lt = tab_layout(X, Y, T, Xp, kKindChunk);
    const double strike = 0.001 * (double)item.strike;  // strikes (:247)
    const int steps = T > 1 ? T - 1 : 0;

    // Cluster peers holding the rows just above / below this CTA's block.
    const S* Aprev = nullptr;
    const S* Anext = nullptr;
    if (!GSTATE && clustered) {
      cg::cluster_group cl = cg::this_cluster();
      if (rank > 0) Aprev = cl.map_shared_rank(A, rank - 1);
      if (rank < C - 1 && r0 + Ycs < Y) Anext = cl.map_shared_rank(A, rank + 1);
    }

    __syncthreads();  // the previous instance is finished with A, B and the tables
    // setPayoff (:46-47) and the column / row constants.
    for (int e = tid; e < Yc * Xp; e += NT) {
      const int jl = e / Xp, i = e - jl * Xp;
      const S v = (i < X) ? (S)fmax(tabc[Lt.x + i] - strike, 0.0) : (S)0;
      A[jl * LD + col_off<S>(i)] = v;
    }
    for (int e = tid; e < 4 * Xp; e += NT) s_colc[e] = (S)tabc[Lt.colc + e];
    for (int e = tid; e < 4 * Yc; e += NT) s_rowc[e] = (S)tabc[Lt.rowc + 4LL * r0 + e];

    auto load_tables = [&](int k, S* tb) {
      for (int jl = tid; jl < Ycs; jl += NT) {
        S e = 0, mY = 0, nY = 0, rb = 0;
        if (jl < Yc) {
          const int jg = r0 + jl;
          e = (S)tabc[Lt.eyt + (int64_t)k * Lt.eyt_ld + jg];
          const double* yc = tabc + Lt.yco + ((int64_t)k * Y + jg) * 4;
          mY = (S)yc[0];
          nY = (S)yc[1];
          rb = (S)yc[2];
        }
        tb[st.eyt + jl] = e;
        tb[st.mY + jl] = mY;
        tb[st.nY + jl] = nY;
        tb[st.rbY + jl] = rb;
      }
      // Within-chunk prefix products of the forward multipliers and suffix
      // products of the backward ones: column- and strike-independent.
      for (int ch = tid; ch < Lf.P; ch += NT) {
        const int jb = ch * kKY, je = min(Yc, jb + kKY);
        S prod = (S)1;
        for (int j = jb; j < je; j++) {
          prod = prod * (S)tabc[Lt.yco + ((int64_t)k * Y + r0 + j) * 4 + 0];
          tb[st.cp + j] = prod;
        }
        tb[st.BF + ch] = prod;
        prod = (S)1;
        for (int j = je - 1; j >= jb; j--) {
          prod = prod * (S)tabc[Lt.yco + ((int64_t)k * Y + r0 + j) * 4 + 1];
          tb[st.cq + j] = prod;
        }
        tb[st.BB + ch] = prod;
      }
    };

    if (steps == 0) {  // numT == 1: no time step, the price is the payoff
      if (tid == 0 && c.yindex >= r0 && c.yindex < r0 + Yc)
        args.out[c.out + item.strike] = fmax(tabc[Lt.x + c.xindex] - strike, 0.0);
      continue;
    }
    load_tables(steps - 1, s_tab[sc & 1]);

    // X-sweep lane geometry: p lanes share one row, KX columns each.
    const int p = Xp / KX;
    const int RW = 32 / p;
    const int q = lane & (p - 1);
    const int rr = lane / p;
    const int i0 = q * KX;
    // Y-sweep geometry: units of 32 columns x kKY rows, one warp each.
    const int G = Lf.G, P = Lf.P, U = Lf.U;

    for (int s = 0; s < steps; s++, sc++) {
      const int k = steps - 1 - s;  // reverse (zip (init tl) (tail tl))  (:217)
      if (clustered) cg::this_cluster().sync(); else __syncthreads();
      if (s + 1 < steps) load_tables(k - 1, s_tab[(sc + 1) & 1]);
      S* tb = s_tab[sc & 1];
      const S dt = (S)tabc[Lt.dtinv + k];
      const S half = (S)0.5;

      // ---------------- explicitX + explicitY + implicitX (row sweep) ----------------
      const PV* pivk = args.piv + c.piv + (int64_t)k * Y * Xp;
      for (int jb = warp * RW; jb < Yc; jb += NW * RW) {
        const int jl = jb + rr;
        const bool vrow = jl < Yc;
        const int jg = r0 + jl;
        S e = 0, g0 = 0, g1 = 0, g2 = 0;
        if (vrow) {
          e = tb[st.eyt + jl];
          g0 = s_rowc[4 * jl + 0];
          g1 = s_rowc[4 * jl + 1];
          g2 = s_rowc[4 * jl + 2];
        }
        S rb[KX];
        load_piv<KX>(pivk + (int64_t)jg * Xp + i0, rb, vrow);
        S R[KX], Up[KX], Dn[KX];
        load_chunk<KX>(A + jl * LD, i0, R, vrow);
        const S* uprow = (jl > 0) ? A + (jl - 1) * LD : (Aprev ? Aprev + (Ycs - 1) * LD : nullptr);
        const S* dnrow = (jl + 1 < Yc) ? A + (jl + 1) * LD : (Anext ? Anext : nullptr);
        load_chunk<KX>(uprow, i0, Up, vrow && uprow != nullptr);
        load_chunk<KX>(dnrow, i0, Dn, vrow && dnrow != nullptr);

        S Rl = __shfl_up_sync(0xffffffffu, R[KX - 1], 1, p);
        S Rr = __shfl_down_sync(0xffffffffu, R[0], 1, p);
        S rbl = __shfl_up_sync(0xffffffffu, rb[KX - 1], 1, p);
        if (q == 0) { Rl = 0; rbl = 0; }
        if (q == p - 1) Rr = 0;

        S V[KX], z[KX], Pm[KX], nn[KX];
        S zl = 0, Pl = 1;
#pragma unroll
        for (int m = 0; m < KX; m++) {
          const int i = i0 + m;
          const S* cc = s_colc + 4 * i;
          const S var = cc[0] * e;  // VarX (:63) = exp(2 beta log x_i) * exp(2 (y_j - nu^2 t / 2))
          const S p0 = var * cc[1], p1 = var * cc[2], p2 = var * cc[3];
          const S left = m ? R[m - 1] : Rl;
          const S right = (m < KX - 1) ? R[m + 1] : Rr;
          const S ex = p0 * left + p1 * R[m] + p2 * right;   // explicitX (:134-145)
          const S v = g0 * Up[m] + g1 * R[m] + g2 * Dn[m];     // explicitY (:199)
          V[m] = v;
          const S u = (dt * R[m] + half * ex) + v;            // :196, :200
          const S rbp = m ? rb[m - 1] : rbl;
          const S mult = half * p0 * rbp;  // -a_i / b'_{i-1}  (:100)
          nn[m] = half * p2 * rb[m];       // -c_i / b'_i      (:116)
          zl = u + mult * zl;
          z[m] = zl;
          Pl = mult * Pl;
          Pm[m] = Pl;
        }
        // forward recurrence across the p lanes of the row (inclusive scan of
        // affine maps z -> A + B z), then fix up with the exclusive prefix.
        S Aa = zl, Bb = Pl;
        for (int d = 1; d < p; d <<= 1) {
          const S Ap = __shfl_up_sync(0xffffffffu, Aa, d, p);
          const S Bp = __shfl_up_sync(0xffffffffu, Bb, d, p);
          if (q >= d) { Aa = Aa + Bb * Ap; Bb = Bb * Bp; }
        }
        S zin = __shfl_up_sync(0xffffffffu, Aa, 1, p);
        if (q == 0) zin = 0;
#pragma unroll
        for (int m = 0; m < KX; m++) z[m] = z[m] + Pm[m] * zin;
        // backward recurrence x_i = z_i / b'_i - (c_i / b'_i) x_{i+1}  (:111-123)
        S xl = 0, Ql = 1;
#pragma unroll
        for (int m = KX - 1; m >= 0; m--) {
          xl = rb[m] * z[m] + nn[m] * xl;
          z[m] = xl;
          Ql = nn[m] * Ql;
          Pm[m] = Ql;
        }
        Aa = xl;
        Bb = Ql;
        for (int d = 1; d < p; d <<= 1) {
          const S An = __shfl_down_sync(0xffffffffu, Aa, d, p);
          const S Bn = __shfl_down_sync(0xffffffffu, Bb, d, p);
          if (q + d < p) { Aa = Aa + Bb * An; Bb = Bb * Bn; }
        }
        S xin = __shfl_down_sync(0xffffffffu, Aa, 1, p);
        if (q == p - 1) xin = 0;
        S Yr[KX];
#pragma unroll
        for (int m = 0; m < KX; m++) {
          const S x = z[m] + Pm[m] * xin;
          Yr[m] = dt * x - half * V[m];  // :205
        }
        if (vrow) store_chunk<KX>(B + jl * LD, i0, Yr);
      }
      __syncthreads();

      // ---------------- implicitY (column sweep) ----------------
      // pass 1: forward recurrence, chunk-local (start value 0), in place in B.
      for (int u = warp; u < U; u += NW) {
        const int g = u / P, ch = u - g * P;
        const int col = g * 32 + lane;
        const bool vc = col < X;
        const int jb = ch * kKY, je = min(Yc, jb + kKY);
        S* Bc = B + col_off<S>(col);
        S zz = 0;
        for (int j = jb; j < je; j++) {
          const S y = vc ? Bc[j * LD] : (S)0;
          zz = y + tb[st.mY + j] * zz;
          if (vc) Bc[j * LD] = zz;
        }
        s_aggF[u * 32 + lane] = zz;
      }
      __syncthreads();
      if (clustered) {
        // fold this CTA's chunks into one block aggregate per column
        for (int col = tid; col < G * 32; col += NT) {
          const int g = col >> 5, ln = col & 31;
          S a = 0;
          for (int ch = 0; ch < P; ch++) a = s_aggF[(g * P + ch) * 32 + ln] + tb[st.BF + ch] * a;
          s_blkF[col] = a;
        }
        if (tid == 0) {
          S b = 1;
          for (int ch = 0; ch < P; ch++) b = tb[st.BF + ch] * b;
          tb[st.blkBF] = b;
        }
        cg::cluster_group cl = cg::this_cluster();
        cl.sync();
        for (int col = tid; col < G * 32; col += NT) {
          S zv = 0;
          for (int r = 0; r < rank; r++) {
            const S* rb = cl.map_shared_rank(s_blkF, r);
            const S* rt = cl.map_shared_rank(tb, r);
            zv = rb[col] + rt[st.blkBF] * zv;
          }
          s_zin[col] = zv;
        }
        __syncthreads();
      }
      // pass 2 (reverse order): forward fix-up, then the backward recurrence
      // chunk-locally (start value 0), in place in B.
      for (int u = warp; u < U; u += NW) {
        const int g = u / P, ch = u - g * P;
        const int col = g * 32 + lane;
        const bool vc = col < X;
        const int jb = ch * kKY, je = min(Yc, jb + kKY);
        S* Bc = B + col_off<S>(col);
        S zin = clustered ? s_zin[g * 32 + lane] : (S)0;
        for (int c2 = 0; c2 < ch; c2++) zin = s_aggF[(g * P + c2) * 32 + lane] + tb[st.BF + c2] * zin;
        S xx = 0;
        for (int j = je - 1; j >= jb; j--) {
          const S zv = (vc ? Bc[j * LD] : (S)0) + tb[st.cp + j] * zin;
          xx = tb[st.rbY + j] * zv + tb[st.nY + j] * xx;
          if (vc) Bc[j * LD] = xx;
        }
        s_aggB[u * 32 + lane] = xx;
      }
      __syncthreads();
      if (clustered) {
        for (int col = tid; col < G * 32; col += NT) {
          const int g = col >> 5, ln = col & 31;
          S a = 0;
          for (int ch = P - 1; ch >= 0; ch--) a = s_aggB[(g * P + ch) * 32 + ln] + tb[st.BB + ch] * a;
          s_blkB[col] = a;
        }
        if (tid == 0) {
          S b = 1;
          for (int ch = P - 1; ch >= 0; ch--) b = tb[st.BB + ch] * b;
          tb[st.blkBB] = b;
        }
        cg::cluster_group cl = cg::this_cluster();
        cl.sync();
        for (int col = tid; col < G * 32; col += NT) {
          S xv = 0;
          for (int r = C - 1; r > rank; r--) {
            const S* rb = cl.map_shared_rank(s_blkB, r);
            const S* rt = cl.map_shared_rank(tb, r);
            xv = rb[col] + rt[st.blkBB] * xv;
          }
          s_xin[col] = xv;
        }
        __syncthreads();
      }
      // pass 3: backward fix-up; the result is the new grid, written to A.
      for (int u = warp; u < U; u += NW) {
        const int g = u / P, ch = u - g * P;
        const int col = g * 32 + lane;
        const bool vc = col < X;
        const int jb = ch * kKY, je = min(Yc, jb + kKY);
        S* Bc = B + col_off<S>(col);
        S* Ac = A + col_off<S>(col);
        S xin = clustered ? s_xin[g * 32 + lane] : (S)0;
        for (int c2 = P - 1; c2 > ch; c2--) xin = s_aggB[(g * P + c2) * 32 + lane] + tb[st.BB + c2] * xin;
        for (int j = jb; j < je; j++) {
          const S xv = (vc ? Bc[j * LD] : (S)0) + tb[st.cq + j] * xin;
          if (vc) {
            Ac[j * LD] = xv;
            if (s == steps - 1 && col == c.xindex && r0 + j == c.yindex)
              args.out[c.out + item.strike] = (double)xv;  // myResult[myYindex, myXindex]
          }
        }
      }
    }
  }
  // No CTA of a cluster may exit while a peer can still read its shared
  // memory (the last step's backward fold reads peers' block aggregates).
  if (clustered) cg::this_cluster().sync();
}

// f64 result -> f32 output array (the f32 entry point computes in f64).
__global__ void lvc_to_f32_kernel(const double* __restrict__ in, float* __restrict__ out, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (float)in[i];
}

}  // namespace lvc
