// Paired line kernel: the full-tile line kernel's algorithm with every
// shared-memory access widened to two adjacent grid columns.
//
// The rollback of finpar/LocVolCalib.fut:180-209 per time step, on an
// X x Ycs block of the grid held in shared memory (one CTA per strike
// instance, or Ycs rows per CTA of a cluster):
//   X sweep  lane = grid row, a warp unit = 32 rows x 16 columns; the lane
//            walks its 16 columns two at a time, reading the grid, the
//            rows above and below and the pivots as 16-byte pairs, and the
//            column weights W0, W1, W2 as pair broadcasts (planar arrays);
//   Y sweep  lane = two adjacent columns, a warp unit = 64 columns x 16
//            rows; every per-row table entry it broadcasts serves both
//            column recurrences, and grid rows move as 16-byte pairs.
// The row stride LD = numX + 2 is 2 mod 4 doubles, so the 32 lanes of a warp
// reading one 16-byte pair from 32 consecutive rows fall into 4 conflict-free
// wavefronts (8 lanes cover the 32 banks), and rows start 16-byte aligned for
// the pair accesses of the Y sweep.  Columns numX and numX + 1 are zero.
// Needs numX % (32 * UPW) == 0 (whole Y units), rows per CTA % 32 == 0 and
// numY = cluster size x rows per CTA.
//
// UPW (units per warp) = 2: each warp owns two X units (two independent
// recurrence chains per lane) and one 64-column Y unit (two columns per lane);
// with UPW = 1 a warp owns one X unit and one 32-column Y unit (one column per
// lane), so the same block runs on twice the warps at half the registers per
// thread -- more warps to hide shared-memory and FP64 latency when the grid's
// shared memory leaves room for only one CTA per SM.
//
// Cluster (C CTAs per instance, rank r holding rows r*Ycs ..): the Y
// recurrences cross the ranks.  Each step, after the forward chunk maps of
// its block are known, a rank pushes them (st.async) to every higher rank and
// folds the lower ranks' maps in rank order into its forward input z_in; the
// same for the backward maps, pushed down and folded from the top into x_in.
// Every wait is on the receiving CTA's own mbarrier, bounded.  The halo rows
// the next step's explicit terms need are computed locally from the folds:
// the row below the block is x_in itself, and the row above is the last row
// of the rank below, x = (1/b') z_in + nY x_first (Thomas backward step with
// that row's forward state z_in and this block's first row x_first).
#pragma once

#include "lvc_line.cuh"

namespace lvc {

struct PairLayout {
  int LD, Ycs, CHx, Ux, CG2, CHy, Uy;
  int bar, barF, barB, A, B, w0, w1, w2, grow, gx, ex, tab0, tab1, tabh, xf, xb, yf, yb, inF, totF, inB, totB,
      zin, xin, total;
};

// Byte offsets of the shared-memory buffers of a CTA holding Ycs rows of an
// X-column grid split over a cluster of C CTAs.  The four mbarriers sit at
// fixed offsets (initialised once per launch, whatever the items).
template <typename S>
LVC_HD PairLayout pair_layout(int X, int Ycs, int upw, int C) {
  PairLayout L;
  auto up = [](int n) { return (n + 15) / 16 * 16; };
  const int s = (int)sizeof(S);
  L.LD = pair_ld(X);
  L.Ycs = Ycs;
  L.CHx = X / kLineK;
  L.Ux = (Ycs / 32) * L.CHx;  // X units: 2 per warp
  L.CG2 = X / (32 * upw);    // column groups of a Y unit (32 * upw columns)
  L.CHy = Ycs / kLineK;
  L.Uy = L.CG2 * L.CHy;       // Y units: 1 per warp
  int o = 0;
  L.bar = o; o += 8;   // bulk copies of the step's pivots and table
  L.barF = o; o += 8;  // cluster: forward chunk maps of the lower ranks have landed
  L.barB = o; o += 16; // cluster: backward chunk maps of the higher ranks have landed
  L.A = o; o += up((Ycs + 2) * L.LD * s);  // rows -1 .. Ycs (halo rows at both ends)
  L.B = o; o += up(Ycs * L.LD * s);
  L.w0 = o; o += up(X * s);               // W_k(i), planar
  L.w1 = o; o += up(X * s);
  L.w2 = o; o += up(X * s);
  L.grow = o; o += up(4 * Ycs * s);        // [Ycs][4] g0..g2 of a row: Y-sweep broadcasts
  L.gx = o; o += up(3 * Ycs * s);          // [3][Ycs] the same, planar: X sweep (lane = row)
  L.ex = o; o += up(Ycs * s);              // [Ycs] e_j of the current step, planar
  L.tab0 = o; o += up(8 * Ycs * 8);
  L.tab1 = o; o += up(8 * Ycs * 8);
  L.tabh = o; o += 2 * 64;                 // cluster: the step-table row above the block, double-buffered
  L.xf = o; o += up(L.Ux / upw * 64 * s);  // [warp][lane] (a, b) of the warps' forward chunk maps
  L.xb = o; o += up(L.Ux / upw * 64 * s);  // the same, backward
  L.yf = o; o += up(L.Uy * 32 * upw * s);
  L.yb = o; o += up(L.Uy * 32 * upw * s);
  // cluster: the chunk maps every other rank pushes here, [rank][column],
  // and the rank's multiplier product (column-independent), [rank]
  const int Cc = C > 1 ? C : 0;
  L.inF = o; o += up(Cc * X * s);
  L.totF = o; o += up(Cc * s);
  L.inB = o; o += up(Cc * X * s);
  L.totB = o; o += up(Cc * s);
  L.zin = o; o += up(X * s);
  L.xin = o; o += up(X * s);
  L.total = o;
  return L;
}

template <typename S> struct P2;
template <> struct P2<double> {
  using T = double2;
  static __device__ __forceinline__ double2 ld(const double* p) { return *reinterpret_cast<const double2*>(p); }
  static __device__ __forceinline__ void st(double* p, double a, double b) {
    *reinterpret_cast<double2*>(p) = make_double2(a, b);
  }
};
template <> struct P2<float> {
  using T = float2;
  static __device__ __forceinline__ float2 ld(const float* p) { return *reinterpret_cast<const float2*>(p); }
  static __device__ __forceinline__ void st(float* p, float a, float b) {
    *reinterpret_cast<float2*>(p) = make_float2(a, b);
  }
};

// N adjacent columns of a row (N = 1 or 2) to and from registers.
template <typename S, int N>
__device__ __forceinline__ void ld_cols(const S* p, S (&v)[N]) {
  if constexpr (N == 2) {
    const auto t = P2<S>::ld(p);
    v[0] = t.x;
    v[1] = t.y;
  } else {
    v[0] = *p;
  }
}
template <typename S, int N>
__device__ __forceinline__ void st_cols(S* p, const S (&v)[N]) {
  if constexpr (N == 2) P2<S>::st(p, v[0], v[1]); else *p = v[0];
}

// Resident CTAs per SM the launch bounds ask for: 256 threads' worth of
// warps, twice that with f32 state (half the shared memory per CTA).
template <typename S, int NT, int UPW> struct PairMinBlocks {
  static constexpr int base = UPW == 2 ? FullMinBlocks<NT>::v : (NT >= 512 ? 1 : 512 / NT);
  static constexpr int v = UPW == 2 && sizeof(S) == 4 ? 2 * base : base;
};

template <typename S, typename PV, int NT, int UPW>
__global__ void __launch_bounds__(NT, (PairMinBlocks<S, NT, UPW>::v)) lvc_line_pair_kernel(RollbackArgs<S, PV> args) {
  constexpr int K = kLineK;
  constexpr int NW = NT / 32;
  constexpr int NU = NW * UPW;  // X units per sweep
  constexpr int UW = 32 * UPW;  // columns per Y unit
  static_assert(UPW == 1 || UPW == 2, "one or two units per warp");
  static_assert(sizeof(S) == sizeof(PV), "pivots are copied verbatim into the state buffer");
  static_assert(K % 2 == 0, "columns are walked in pairs");
  using V = P2<S>;
  constexpr int FB = 2;  // warp maps loaded at once in the X folds
  extern __shared__ __align__(16) unsigned char smem[];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int C = args.C;
  const bool clustered = C > 1;
  int rank = 0;
  if (clustered) rank = (int)cg::this_cluster().block_rank();
  const int cid = blockIdx.x / C, ncl = gridDim.x / C;
  unsigned sc = 0, phase = 0;
  unsigned phF = 0, phB = 0;  // parities of the cluster barriers (one completion per use)
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem);
  uint64_t* barF = bar + 1;
  uint64_t* barB = bar + 2;
  if (tid == 0) {
    mbar_init(bar, 1);
    mbar_init(barF, 1);
    mbar_init(barB, 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();

  for (int it = cid; it < args.n_items; it += ncl) {
    const Item item = args.items[it];
    const CalibDev c = args.calibs[item.calib];
    const int X = c.numX, Y = c.numY, T = c.numT;
    const int Ycs = c.Ycs;
    const int r0 = rank * Ycs;
    const PairLayout Ls = pair_layout<S>(X, Ycs, UPW, C);
    // uniform over the cluster (every CTA of a cluster sees the same item)
    if (c.kind != kKindLine || c.C != C || c.ld != Ls.LD || Ls.total > args.smem_elems * (int)sizeof(S) ||
        Ls.Ux != NU || Ls.Uy != NW || (X % UW) || (Ls.CHx % UPW) || (Ycs % 32) || Ycs * C != Y) {
      if (tid == 0) atomicExch(args.err, 5);
      continue;
    }
    const int LD = Ls.LD;
    S* A = reinterpret_cast<S*>(smem + Ls.A);  // row r of the block at A + (r + 1) * LD
    S* B = reinterpret_cast<S*>(smem + Ls.B);
    S* sW0 = reinterpret_cast<S*>(smem + Ls.w0);
    S* sW1 = reinterpret_cast<S*>(smem + Ls.w1);
    S* sW2 = reinterpret_cast<S*>(smem + Ls.w2);
    S* sG = reinterpret_cast<S*>(smem + Ls.grow);
    S* sGx = reinterpret_cast<S*>(smem + Ls.gx);
    S* sE = reinterpret_cast<S*>(smem + Ls.ex);
    double* const sT0 = reinterpret_cast<double*>(smem + Ls.tab0);
    double* const sT1 = reinterpret_cast<double*>(smem + Ls.tab1);
    S* xf = reinterpret_cast<S*>(smem + Ls.xf);
    S* xb = reinterpret_cast<S*>(smem + Ls.xb);
    S* yf = reinterpret_cast<S*>(smem + Ls.yf);
    S* yb = reinterpret_cast<S*>(smem + Ls.yb);
    S* inF = reinterpret_cast<S*>(smem + Ls.inF);
    S* totF = reinterpret_cast<S*>(smem + Ls.totF);
    S* inB = reinterpret_cast<S*>(smem + Ls.inB);
    S* totB = reinterpret_cast<S*>(smem + Ls.totB);
    double* const sTh = reinterpret_cast<double*>(smem + Ls.tabh);
    S* s_zin = reinterpret_cast<S*>(smem + Ls.zin);
    S* s_xin = reinterpret_cast<S*>(smem + Ls.xin);
    const double* tabc = args.tabs + c.tab;
    const TabLayout Lt = tab_layout(X, Y, T, c.Xp, kKindLine);
    const double strike = 0.001 * (double)item.strike;  // strikes (:247)
    const int steps = T > 1 ? T - 1 : 0;
    const PV* piv = args.piv + c.piv;
    const int64_t Y4 = round4(Y);
    // Cluster pushes (st.async into the other ranks' shared memory, counted
    // on their barriers): this rank's forward block maps go to every higher
    // rank, its backward ones to every lower rank, at slot `rank` -- two
    // exchanges per step.  The halo rows are not exchanged: each rank computes
    // its own from the folds' results (see the fix-up).
    const bool has_prev = clustered && rank > 0, has_next = clustered && rank < C - 1;
    const unsigned fold_bytes_F = (unsigned)(rank * (X + 1) * (int)sizeof(S));
    const unsigned fold_bytes_B = clustered ? (unsigned)((C - 1 - rank) * (X + 1) * (int)sizeof(S)) : 0u;

    // The previous instance is done with every buffer, and -- across the
    // cluster -- every rank has read the last block maps this CTA pushed to it.
    if (clustered) cg::this_cluster().sync(); else __syncthreads();
    // setPayoff (:46-47) on the block and the halo rows (zero at the global
    // boundary and in the two padding columns)
    for (int e = tid; e < (Ycs + 2) * LD; e += NT) {
      const int r = e / LD, i = e - r * LD;
      const bool boundary = (r == 0 && rank == 0) || (r == Ycs + 1 && rank == C - 1);
      A[e] = (i < X && !boundary) ? (S)fmax(tabc[Lt.x + i] - strike, 0.0) : (S)0;
    }
    for (int e = tid; e < 3 * X; e += NT) {
      const int k = e / X, i = e - k * X;
      (k == 0 ? sW0 : k == 1 ? sW1 : sW2)[i] = (S)tabc[Lt.wcol + k * (int64_t)((X + 1) & ~1) + i];
    }
    for (int e = tid; e < 4 * Ycs; e += NT) sG[e] = (S)tabc[Lt.rowc + 4LL * r0 + e];
    // Row constants read with lane = row are planar, so that 32 rows fall in
    // distinct banks (the [row][4] and [row][8] layouts would conflict 8- and
    // 16-way).
    for (int e = tid; e < 3 * Ycs; e += NT) {
      const int k = e / Ycs, j = e - k * Ycs;
      sGx[e] = (S)tabc[Lt.rowc + 4LL * (r0 + j) + k];
    }

    if (steps == 0) {
      if (tid == 0 && c.yindex >= r0 && c.yindex < r0 + Ycs)
        args.out[c.out + item.strike] = fmax(tabc[Lt.x + c.xindex] - strike, 0.0);
      continue;
    }
    const unsigned piv_bytes = (unsigned)(Ycs * LD * (int)sizeof(S));  // a multiple of 16
    const unsigned tab_bytes = (unsigned)(Ycs * 64);
    const unsigned tabh_bytes = has_prev ? 64u : 0u;
    auto issue_copies = [&](int k, unsigned buf) {
      if (tid == 0) {
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        mbar_expect_tx(bar, piv_bytes + tab_bytes + tabh_bytes);
        bulk_g2s(B, piv + ((int64_t)k * Y4 + r0) * LD, piv_bytes, bar);
        bulk_g2s(buf ? sT1 : sT0, tabc + Lt.stab + ((int64_t)k * Y + r0) * 8, tab_bytes, bar);
        if (has_prev) bulk_g2s(sTh + 8 * buf, tabc + Lt.stab + ((int64_t)k * Y + r0 - 1) * 8, 64, bar);
      }
    };
    issue_copies(steps - 1, sc & 1);

    // X units u = UPW * warp + q: rows rgx*32 + lane, columns chx*16 .. -- a
    // warp's two units are neighbouring chunks of the same rows (the number of
    // chunks per row, numX / 16, is even), so the second unit's chunk prefix
    // is the first one's plus one chunk
    int rgx[UPW], chx[UPW], jl[UPW];
#pragma unroll
    for (int q = 0; q < UPW; q++) {
      const int u = UPW * warp + q;
      rgx[q] = u / Ls.CHx;
      chx[q] = u - rgx[q] * Ls.CHx;
      jl[q] = rgx[q] * 32 + lane;
    }
    // A warp's units are consecutive chunks of one row group (numX / 16 is a
    // multiple of UPW), so the warp composes their chunk maps in registers and
    // publishes one map per warp; a warp then folds the maps of the warps
    // before it (forward) or after it (backward) in its row group.
    const int WPG = Ls.CHx / UPW;           // warps per row group
    const int wg0 = (warp / WPG) * WPG;     // first warp of this warp's row group
    // Y unit u = warp: columns cgy*UW + UPW*lane (+ h < UPW), rows chy*16 ..
    const int cgy = warp / Ls.CHy, chy = warp - cgy * Ls.CHy;
    const int col0 = cgy * UW + UPW * lane;
    // output lane: the column and element holding myResult[myYindex, myXindex]
    int out_h = -1, out_m = 0;
    {
      const int jy = c.yindex - r0 - chy * K;
      if (c.xindex >= col0 && c.xindex < col0 + UPW && jy >= 0 && jy < K) {
        out_h = c.xindex - col0;
        out_m = jy;
      }
    }

    bool timed_out = false;  // a bulk-copy wait of this item gave up
    for (int s = 0; s < steps; s++, sc++) {
      const int k = steps - 1 - s;
      if (!mbar_wait(bar, phase, timed_out ? kWaitPollsAfterTimeout : kWaitPolls)) {
        timed_out = true;
        atomicExch(args.err, 3);
      }
      phase ^= 1u;
      const double* tb = (sc & 1) ? sT1 : sT0;
      // e_j of this step, planar (the barrier below orders it before the X
      // sweep; its last readers were the previous step's passes 1 and 2)
      for (int j = tid; j < Ycs; j += NT) sE[j] = (S)tb[j * 8 + kSlotE];
      __syncthreads();
      const S dt = (S)tabc[Lt.dtinv + k];

      // -------- X sweep pass 1: explicitX + explicitY, forward recurrence (chunk-local) --------
      S z[UPW][K], PQ[UPW][K];
      S zl[UPW], Pl[UPW];  // each unit's forward chunk map: z_end = zl + Pl * z_in
      {
        S e[UPW], g0[UPW], g1[UPW], g2[UPW], Rl[UPW], rbp[UPW];
        typename V::T Rc[UPW];
#pragma unroll
        for (int q = 0; q < UPW; q++) {
          const int ib = chx[q] * K;
          const S* Arow = A + (jl[q] + 1) * LD;
          e[q] = sE[jl[q]];
          g0[q] = sGx[jl[q]];
          g1[q] = sGx[Ycs + jl[q]];
          g2[q] = sGx[2 * Ycs + jl[q]];
          Rl[q] = ib > 0 ? Arow[ib - 1] : (S)0;
          Rc[q] = V::ld(Arow + ib);
          rbp[q] = ib > 0 ? B[jl[q] * LD + ib - 1] : (S)0;
          zl[q] = 0;
          Pl[q] = 1;
        }
#pragma unroll
        for (int p = 0; p < K / 2; p++) {
#pragma unroll
          for (int q = 0; q < UPW; q++) {
            const int i = chx[q] * K + 2 * p;
            const S* Arow = A + (jl[q] + 1) * LD;
            const auto Rn = V::ld(Arow + i + 2);   // columns i+2, i+3 (numX, numX+1 are zero)
            const auto up = V::ld(Arow + i - LD);  // rows j-1 and j+1 (halo rows at the block edges)
            const auto dn = V::ld(Arow + i + LD);
            const auto w0 = V::ld(sW0 + i);
            const auto w1 = V::ld(sW1 + i);
            const auto w2 = V::ld(sW2 + i);
            const auto rb = V::ld(B + jl[q] * LD + i);
            {  // column i
              const S v = g0[q] * up.x + g1[q] * Rc[q].x + g2[q] * dn.x;    // explicitY (:199)
              const S sx = w0.x * Rl[q] + w1.x * Rc[q].x + w2.x * Rc[q].y;   // explicitX / (0.5 e)
              const S u = e[q] * sx + (dt * Rc[q].x + v);                    // :195-200
              const S mult = (e[q] * w0.x) * rbp[q];                         // -a_i / b'_{i-1}
              zl[q] = u + mult * zl[q];
              Pl[q] = mult * Pl[q];
              z[q][2 * p] = zl[q];
              PQ[q][2 * p] = Pl[q];
            }
            {  // column i + 1
              const S v = g0[q] * up.y + g1[q] * Rc[q].y + g2[q] * dn.y;
              const S sx = w0.y * Rc[q].x + w1.y * Rc[q].y + w2.y * Rn.x;
              const S u = e[q] * sx + (dt * Rc[q].y + v);
              const S mult = (e[q] * w0.y) * rb.x;
              zl[q] = u + mult * zl[q];
              Pl[q] = mult * Pl[q];
              z[q][2 * p + 1] = zl[q];
              PQ[q][2 * p + 1] = Pl[q];
            }
            rbp[q] = rb.y;
            Rl[q] = Rc[q].y;
            Rc[q] = Rn;
          }
        }
        // the warp's map (unit 1 after unit 0)
        if constexpr (UPW == 2)
          V::st(xf + (warp * 32 + lane) * 2, zl[1] + Pl[1] * zl[0], Pl[1] * Pl[0]);
        else
          V::st(xf + (warp * 32 + lane) * 2, zl[0], Pl[0]);
      }
      __syncthreads();
      // -------- pass 2: forward fix-up, backward recurrence (chunk-local) --------
      S xl[UPW], Ql[UPW];  // each unit's backward chunk map: x_start = xl + Ql * x_in
      {
        S zin[UPW], e[UPW];
        {
          S a = 0;
          // the maps of the warps before this one, in order; loads in batches
          // of FB so that their latencies overlap
          for (int w0 = wg0; w0 < warp; w0 += FB) {
            typename V::T f[FB];
#pragma unroll
            for (int t = 0; t < FB; t++)
              if (w0 + t < warp) f[t] = V::ld(xf + ((w0 + t) * 32 + lane) * 2);
#pragma unroll
            for (int t = 0; t < FB; t++)
              if (w0 + t < warp) a = f[t].x + f[t].y * a;
          }
          zin[0] = a;
          if constexpr (UPW == 2) zin[1] = zl[0] + Pl[0] * a;
        }
#pragma unroll
        for (int q = 0; q < UPW; q++) {
          xl[q] = 0;
          Ql[q] = 1;
          e[q] = sE[jl[q]];
        }
#pragma unroll
        for (int p = K / 2 - 1; p >= 0; p--) {
#pragma unroll
          for (int q = 0; q < UPW; q++) {
            const int i = chx[q] * K + 2 * p;
            const auto rb = V::ld(B + jl[q] * LD + i);
            const auto w2 = V::ld(sW2 + i);
            {  // column i + 1
              const S zz = z[q][2 * p + 1] + PQ[q][2 * p + 1] * zin[q];
              const S aR = e[q] * w2.y;
              xl[q] = rb.y * (zz + aR * xl[q]);  // x_i = (z_i - c_i x_{i+1}) / b'_i
              Ql[q] = (aR * rb.y) * Ql[q];
              z[q][2 * p + 1] = xl[q];
              PQ[q][2 * p + 1] = Ql[q];
            }
            {  // column i
              const S zz = z[q][2 * p] + PQ[q][2 * p] * zin[q];
              const S aR = e[q] * w2.x;
              xl[q] = rb.x * (zz + aR * xl[q]);
              Ql[q] = (aR * rb.x) * Ql[q];
              z[q][2 * p] = xl[q];
              PQ[q][2 * p] = Ql[q];
            }
          }
        }
        // the warp's backward map (unit 0 before unit 1)
        if constexpr (UPW == 2)
          V::st(xb + (warp * 32 + lane) * 2, xl[0] + Ql[0] * xl[1], Ql[0] * Ql[1]);
        else
          V::st(xb + (warp * 32 + lane) * 2, xl[0], Ql[0]);
      }
      __syncthreads();
      // -------- pass 3: backward fix-up; dtInv * u goes to B (:205) --------
      {
        S xin[UPW];
        {
          S a = 0;
          // the maps of the warps after this one, from the last one down
          const int wl = wg0 + WPG - 1;
          for (int w0 = wl; w0 > warp; w0 -= FB) {
            typename V::T f[FB];
#pragma unroll
            for (int t = 0; t < FB; t++)
              if (w0 - t > warp) f[t] = V::ld(xb + ((w0 - t) * 32 + lane) * 2);
#pragma unroll
            for (int t = 0; t < FB; t++)
              if (w0 - t > warp) a = f[t].x + f[t].y * a;
          }
          xin[UPW - 1] = a;
          if constexpr (UPW == 2) xin[0] = xl[1] + Ql[1] * a;
        }
#pragma unroll
        for (int p = 0; p < K / 2; p++) {
#pragma unroll
          for (int q = 0; q < UPW; q++) {
            const int i = chx[q] * K + 2 * p;
            V::st(B + jl[q] * LD + i, dt * (z[q][2 * p] + PQ[q][2 * p] * xin[q]),
                  dt * (z[q][2 * p + 1] + PQ[q][2 * p + 1] * xin[q]));
          }
        }
      }
      __syncthreads();

      // -------- Y sweep: lane = columns col0 .. col0 + UPW - 1 --------
      S y[UPW][K];
      {
        S zz[UPW], Ru[UPW], Rm[UPW];
        const int j0 = chy * K;
        ld_cols<S, UPW>(A + j0 * LD + col0, Ru);        // row j0 - 1 (halo row at the block edge)
        ld_cols<S, UPW>(A + (j0 + 1) * LD + col0, Rm);  // row j0
#pragma unroll
        for (int h = 0; h < UPW; h++) zz[h] = 0;
#pragma unroll
        for (int m = 0; m < K; m++) {
          const int j = j0 + m;
          S Rd[UPW], bx[UPW];
          ld_cols<S, UPW>(A + (j + 2) * LD + col0, Rd);  // row j + 1
          ld_cols<S, UPW>(B + j * LD + col0, bx);
          const auto g01 = V::ld(sG + 4 * j);
          const S g2 = sG[4 * j + 2];
          const S my = (S)tb[j * 8 + kSlotMY];
#pragma unroll
          for (int h = 0; h < UPW; h++) {
            const S v = g01.x * Ru[h] + g01.y * Rm[h] + g2 * Rd[h];  // explicitY (:199)
            zz[h] = (bx[h] - (S)0.5 * v) + my * zz[h];              // :205, forward recurrence
            y[h][m] = zz[h];
            Ru[h] = Rm[h];
            Rm[h] = Rd[h];
          }
        }
        st_cols<S, UPW>(yf + warp * UW + UPW * lane, zz);
      }
      __syncthreads();
      if (s + 1 < steps) issue_copies(k - 1, (sc + 1) & 1);
      if (clustered) {
        // this rank's forward block map of each column, pushed to every
        // higher rank; then the lower ranks' maps, folded in rank order
        for (int col = tid; col < X; col += NT) {
          const int g = col / UW, w = col - g * UW;
          S a = 0;
          for (int c2 = 0; c2 < Ls.CHy; c2++)
            a = yf[(g * Ls.CHy + c2) * UW + w] + (S)tb[(c2 * K + K - 1) * 8 + kSlotCP] * a;
          for (int h = rank + 1; h < C; h++)
            st_async(cluster_addr(inF + rank * X + col, h), a, cluster_addr(barF, h));
        }
        if (tid == 0) {
          S b = 1;
          for (int c2 = 0; c2 < Ls.CHy; c2++) b = (S)tb[(c2 * K + K - 1) * 8 + kSlotCP] * b;
          for (int h = rank + 1; h < C; h++) st_async(cluster_addr(totF + rank, h), b, cluster_addr(barF, h));
          mbar_expect_tx(barF, fold_bytes_F);
        }
        if (!mbar_wait_cluster(barF, phF, timed_out ? kWaitPollsAfterTimeout : kWaitPolls)) {
          timed_out = true;
          atomicExch(args.err, 3);
        }
        phF ^= 1u;
        for (int col = tid; col < X; col += NT) {
          S zv = 0;
          for (int q = 0; q < rank; q++) zv = inF[q * X + col] + totF[q] * zv;
          s_zin[col] = zv;
        }
        __syncthreads();
      }
      {
        S zin[UPW], xx[UPW];
#pragma unroll
        for (int h = 0; h < UPW; h++) {
          zin[h] = 0;
          xx[h] = 0;
        }
        if (clustered) ld_cols<S, UPW>(s_zin + col0, zin);
        for (int c2 = 0; c2 < chy; c2++) {
          S a[UPW];
          ld_cols<S, UPW>(yf + (cgy * Ls.CHy + c2) * UW + UPW * lane, a);
          const S cp = (S)tb[(c2 * K + K - 1) * 8 + kSlotCP];
#pragma unroll
          for (int h = 0; h < UPW; h++) zin[h] = a[h] + cp * zin[h];
        }
#pragma unroll
        for (int m = K - 1; m >= 0; m--) {
          const int j = chy * K + m;
          const double2 nr = *reinterpret_cast<const double2*>(tb + j * 8 + kSlotNY);  // nY, 1/b'
          const S cp = (S)tb[j * 8 + kSlotCP];
#pragma unroll
          for (int h = 0; h < UPW; h++) {
            const S zv = y[h][m] + cp * zin[h];
            xx[h] = (S)nr.y * zv + (S)nr.x * xx[h];
            y[h][m] = xx[h];
          }
        }
        st_cols<S, UPW>(yb + warp * UW + UPW * lane, xx);
      }
      __syncthreads();
      if (clustered) {
        // the same for the backward maps: pushed to every lower rank, the
        // higher ranks' folded from the top rank down
        for (int col = tid; col < X; col += NT) {
          const int g = col / UW, w = col - g * UW;
          S a = 0;
          for (int c2 = Ls.CHy - 1; c2 >= 0; c2--)
            a = yb[(g * Ls.CHy + c2) * UW + w] + (S)tb[(c2 * K) * 8 + kSlotCQ] * a;
          for (int h = 0; h < rank; h++)
            st_async(cluster_addr(inB + rank * X + col, h), a, cluster_addr(barB, h));
        }
        if (tid == 0) {
          S b = 1;
          for (int c2 = Ls.CHy - 1; c2 >= 0; c2--) b = (S)tb[(c2 * K) * 8 + kSlotCQ] * b;
          for (int h = 0; h < rank; h++) st_async(cluster_addr(totB + rank, h), b, cluster_addr(barB, h));
          mbar_expect_tx(barB, fold_bytes_B);
        }
        if (!mbar_wait_cluster(barB, phB, timed_out ? kWaitPollsAfterTimeout : kWaitPolls)) {
          timed_out = true;
          atomicExch(args.err, 3);
        }
        phB ^= 1u;
        for (int col = tid; col < X; col += NT) {
          S xv = 0;
          for (int q = C - 1; q > rank; q--) xv = inB[q * X + col] + totB[q] * xv;
          s_xin[col] = xv;
        }
        __syncthreads();
      }
      {
        S xin[UPW];
#pragma unroll
        for (int h = 0; h < UPW; h++) xin[h] = 0;
        if (clustered) ld_cols<S, UPW>(s_xin + col0, xin);
        for (int c2 = Ls.CHy - 1; c2 > chy; c2--) {
          S b[UPW];
          ld_cols<S, UPW>(yb + (cgy * Ls.CHy + c2) * UW + UPW * lane, b);
          const S cq = (S)tb[(c2 * K) * 8 + kSlotCQ];
#pragma unroll
          for (int h = 0; h < UPW; h++) xin[h] = b[h] + cq * xin[h];
        }
#pragma unroll
        for (int m = 0; m < K; m++) {
          const int j = chy * K + m;
          const S cq = (S)tb[j * 8 + kSlotCQ];
          S xv[UPW];
#pragma unroll
          for (int h = 0; h < UPW; h++) {
            xv[h] = y[h][m] + cq * xin[h];
            y[h][m] = xv[h];
          }
          st_cols<S, UPW>(A + (j + 1) * LD + col0, xv);
        }
        // Cluster halo rows for the next step, computed here: the row below
        // the block is the first row of the rank above, which is this rank's
        // x_in; the row above is the last row of the rank below,
        // x = (1/b') z_in + nY x_first, with z_in this rank's forward input
        // (the forward state of that row) and x_first this block's first row.
        if (has_prev && chy == 0) {
          const double* th = sTh + 8 * (sc & 1);
          const S rbh = (S)th[kSlotRB], nyh = (S)th[kSlotNY];
          S zr[UPW], t[UPW];
          ld_cols<S, UPW>(s_zin + col0, zr);
#pragma unroll
          for (int h = 0; h < UPW; h++) t[h] = rbh * zr[h] + nyh * y[h][0];
          st_cols<S, UPW>(A + col0, t);
        }
        if (has_next && chy == Ls.CHy - 1) st_cols<S, UPW>(A + (Ycs + 1) * LD + col0, xin);
        if (s == steps - 1 && out_h >= 0) {
          S pv = 0;
#pragma unroll
          for (int h = 0; h < UPW; h++)
#pragma unroll
            for (int m = 0; m < K; m++)
              if (h == out_h && m == out_m) pv = y[h][m];
          args.out[c.out + item.strike] = (double)pv;  // myResult[myYindex, myXindex]
        }
      }
    }
  }
  if (clustered) cg::this_cluster().sync();
}

}  // namespace lvc
