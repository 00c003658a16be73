// Line kernel: the rollback of finpar/LocVolCalib.fut:180-236 with one grid
// line per lane in both sweeps.
//
// X sweep (explicitX + explicitY + implicitX, :195-202): a warp owns 32
//   consecutive rows and a chunk of kLineK columns; lane j walks row j
//   left to right.  The row neighbours are the lane's own previous/next
//   values, the column neighbours (rows j-1, j+1) arrive by warp shuffle, and
//   the per-column constants are warp-wide broadcasts.  The X pivots 1/b'_i
//   of the step (strike-independent, built by the pivot kernel) sit in the B
//   buffer, where a TMA bulk copy put them during the previous step.  The two
//   linear recurrences of tridagPar (:96-123) run chunk-locally in registers;
//   chunk aggregates are combined across the warps of a row group through
//   shared memory.
// Y sweep (implicitY, :204-209): a warp owns 32 consecutive columns and a
//   chunk of kLineK rows; lane i walks column i.  Multipliers are per-row
//   broadcasts from the step table; chunks combine across warps and, when the
//   grid is split over a thread-block cluster, across CTAs through
//   distributed shared memory.
//
// Every shared-memory access of the grid is conflict-free: rows have an odd
// stride, so 32 lanes reading one column (X sweep) or one row (Y sweep) hit
// 32 distinct 8-byte bank pairs.
#pragma once
#include "lvc_kernels.cuh"

namespace lvc {

// Shared-memory carve-up (byte offsets, 16-byte aligned) for a CTA holding
// Ycs rows of an X-column grid with NW warps.
struct LineLayout {
  int LD, Ycs, RGx, CHx, Ux, CGy, CHy, Uy, xa;
  int A, B, wcol, grow, tab0, tab1, xfa, xfb, xba, xbb, yf, yb, blkF, blkB, zin, xin, tot, bar, total;
};

template <typename S>
LVC_HD LineLayout line_layout(int X, int Ycs, int NW) {
  LineLayout L;
  auto up = [](int n) { return (n + 15) / 16 * 16; };
  const int s = (int)sizeof(S);
  L.LD = line_ld(X);  // odd stride: conflict-free column access
  L.Ycs = Ycs;
  L.RGx = ceil_div(Ycs, 32);
  L.CHx = ceil_div(X, kLineK);
  L.Ux = L.RGx * L.CHx;
  L.CGy = ceil_div(X, 32);
  L.CHy = ceil_div(Ycs, kLineK);
  L.Uy = L.CGy * L.CHy;
  L.xa = (X + 1) & ~1;
  int o = 0;
  L.bar = o; o += 16;  // fixed location: initialised once per kernel launch
  L.A = o; o += up(Ycs * L.LD * s);
  L.B = o; o += up(Ycs * L.LD * s + 16);  // + room for a bulk copy rounded up to 16 bytes
  L.wcol = o; o += up(3 * L.xa * s);
  L.grow = o; o += up(4 * Ycs * s);
  L.tab0 = o; o += up(8 * Ycs * 8);
  L.tab1 = o; o += up(8 * Ycs * 8);
  L.xfa = o; o += up(NW * 32 * s);
  L.xfb = o; o += up(NW * 32 * s);
  L.xba = o; o += up(NW * 32 * s);
  L.xbb = o; o += up(NW * 32 * s);
  L.yf = o; o += up(NW * 32 * s);
  L.yb = o; o += up(NW * 32 * s);
  L.blkF = o; o += up(L.CGy * 32 * s);
  L.blkB = o; o += up(L.CGy * 32 * s);
  L.zin = o; o += up(L.CGy * 32 * s);
  L.xin = o; o += up(L.CGy * 32 * s);
  L.tot = o; o += up(4 * s);
  L.total = o;
  return L;
}

// ---- mbarrier + bulk copy (TMA, no multicast) ----
__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
  unsigned done;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(done)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return done != 0;
}
// Bounded wait: gives up after `limit` polls (each poll may suspend the
// thread for a while); the caller flags an error instead of hanging the GPU.
// After a first timeout the kernels pass a short limit for the rest of the
// item, so a copy that never lands costs one long wait, not one per step.
constexpr int kWaitPolls = 1 << 22;
constexpr int kWaitPollsAfterTimeout = 64;
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity, int limit = kWaitPolls) {
  for (int i = 0; i < limit; i++)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// ---- pushes to another CTA of the cluster (distributed shared memory) ----
// The address of `p` (a shared-memory location of this CTA) in the shared
// window of cluster rank `rank`: every CTA of a launch has the same layout,
// so the same offset names the same buffer there.
__device__ __forceinline__ unsigned cluster_addr(const void* p, int rank) {
  unsigned r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;\n" : "=r"(r) : "r"(smem_u32(p)), "r"(rank));
  return r;
}
// st.async: stores into a remote CTA's shared memory and counts the bytes on
// that CTA's mbarrier (complete_tx, release at cluster scope), so the
// receiver learns of the data by its own barrier -- no cluster barrier.
__device__ __forceinline__ void st_async(unsigned dst, double v, unsigned bar) {
  asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.b64 [%0], %1, [%2];\n" ::"r"(dst),
               "l"(__double_as_longlong(v)), "r"(bar)
               : "memory");
}
__device__ __forceinline__ void st_async(unsigned dst, float v, unsigned bar) {
  asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.b32 [%0], %1, [%2];\n" ::"r"(dst),
               "r"(__float_as_uint(v)), "r"(bar)
               : "memory");
}
__device__ __forceinline__ void st_async2(unsigned dst, double a, double b, unsigned bar) {
  asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.v2.b64 [%0], {%1, %2}, [%3];\n" ::"r"(dst),
               "l"(__double_as_longlong(a)), "l"(__double_as_longlong(b)), "r"(bar)
               : "memory");
}
__device__ __forceinline__ void st_async2(unsigned dst, float a, float b, unsigned bar) {
  asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.v2.b32 [%0], {%1, %2}, [%3];\n" ::"r"(dst),
               "r"(__float_as_uint(a)), "r"(__float_as_uint(b)), "r"(bar)
               : "memory");
}
// Wait for a barrier that remote st.async pushes complete: acquire at cluster
// scope, so the pushed data are visible after it.  Bounded like mbar_wait.
__device__ __forceinline__ bool mbar_try_wait_cluster(uint64_t* bar, unsigned parity) {
  unsigned done;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(done)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return done != 0;
}
__device__ __forceinline__ bool mbar_wait_cluster(uint64_t* bar, unsigned parity, int limit = kWaitPolls) {
  for (int i = 0; i < limit; i++)
    if (mbar_try_wait_cluster(bar, parity)) return true;
  return false;
}

template <typename S, typename PV, int NT>
__global__ void __launch_bounds__(NT, (NT >= 512 ? 1 : 512 / NT)) lvc_line_kernel(RollbackArgs<S, PV> args) {
  constexpr int K = kLineK;
  constexpr int NW = NT / 32;
  constexpr unsigned FULL = 0xffffffffu;
  static_assert(sizeof(S) == sizeof(PV), "pivots are copied verbatim into the state buffer");
  extern __shared__ __align__(16) unsigned char smem[];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int C = args.C;
  const bool clustered = C > 1;
  int rank = 0;
  if (clustered) rank = (int)cg::this_cluster().block_rank();
  const int cid = blockIdx.x / C, ncl = gridDim.x / C;
  unsigned sc = 0;      // running step counter: parity of the double-buffered step tables
  unsigned phase = 0;   // parity of the bulk-copy barrier (one completion per step)
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem);
  if (tid == 0) {
    mbar_init(bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();

  for (int it = cid; it < args.n_items; it += ncl) {
    const Item item = args.items[it];
    const CalibDev c = args.calibs[item.calib];
    const int X = c.numX, Y = c.numY, T = c.numT;
    const int Ycs = c.Ycs;
    const int r0 = rank * Ycs;
    const int Yc = max(0, min(Ycs, Y - r0));
    const LineLayout Ls = line_layout<S>(X, Ycs, NW);
    // uniform over the cluster (every CTA of a cluster sees the same item)
    if (c.kind != kKindLine || c.C != C || c.ld != Ls.LD || Ls.total > args.smem_elems * (int)sizeof(S) ||
        Ls.Ux > NW || Ls.Uy > NW || Yc < 1 || (C > 1 && (Ycs & 3))) {
      if (tid == 0) atomicExch(args.err, 2);
      continue;
    }
    const int LD = Ls.LD;
    S* A = reinterpret_cast<S*>(smem + Ls.A);
    S* B = reinterpret_cast<S*>(smem + Ls.B);
    S* sW = reinterpret_cast<S*>(smem + Ls.wcol);
    S* sG = reinterpret_cast<S*>(smem + Ls.grow);
    double* sT[2] = {reinterpret_cast<double*>(smem + Ls.tab0), reinterpret_cast<double*>(smem + Ls.tab1)};
    S* xfa = reinterpret_cast<S*>(smem + Ls.xfa);
    S* xfb = reinterpret_cast<S*>(smem + Ls.xfb);
    S* xba = reinterpret_cast<S*>(smem + Ls.xba);
    S* xbb = reinterpret_cast<S*>(smem + Ls.xbb);
    S* yf = reinterpret_cast<S*>(smem + Ls.yf);
    S* yb = reinterpret_cast<S*>(smem + Ls.yb);
    S* blkF = reinterpret_cast<S*>(smem + Ls.blkF);
    S* blkB = reinterpret_cast<S*>(smem + Ls.blkB);
    S* s_zin = reinterpret_cast<S*>(smem + Ls.zin);
    S* s_xin = reinterpret_cast<S*>(smem + Ls.xin);
    S* s_tot = reinterpret_cast<S*>(smem + Ls.tot);
    const double* tabc = args.tabs + c.tab;
    const TabLayout Lt = tab_layout(X, Y, T, c.Xp, kKindLine);
    const double strike = 0.001 * (double)item.strike;  // strikes (:247)
    const int steps = T > 1 ? T - 1 : 0;
    const PV* piv = args.piv + c.piv;
    const int64_t Y4 = round4(Y);

    const S* Aprev = nullptr;
    const S* Anext = nullptr;
    if (clustered) {
      cg::cluster_group cl = cg::this_cluster();
      if (rank > 0) Aprev = cl.map_shared_rank(A, rank - 1);
      if (rank < C - 1 && r0 + Ycs < Y) Anext = cl.map_shared_rank(A, rank + 1);
    }

    __syncthreads();  // the previous instance is done with every buffer
    // setPayoff (:46-47), column and row constants
    for (int e = tid; e < Yc * X; e += NT) {
      const int jl = e / X, i = e - jl * X;
      A[jl * LD + i] = (S)fmax(tabc[Lt.x + i] - strike, 0.0);
    }
    for (int e = tid; e < 3 * Ls.xa; e += NT) sW[e] = (S)tabc[Lt.wcol + e];
    for (int e = tid; e < 4 * Yc; e += NT) sG[e] = (S)tabc[Lt.rowc + 4LL * r0 + e];

    if (steps == 0) {  // numT == 1: the price is the payoff
      if (tid == 0 && c.yindex >= r0 && c.yindex < r0 + Yc)
        args.out[c.out + item.strike] = fmax(tabc[Lt.x + c.xindex] - strike, 0.0);
      continue;
    }

    // One thread issues the step's two bulk copies: the pivot rows into B and
    // the step table into sT[buf]; both complete on `bar`.
    const unsigned piv_bytes = (unsigned)((Yc * LD * (int)sizeof(S) + 15) & ~15);
    const unsigned tab_bytes = (unsigned)(Yc * 64);
    auto issue_copies = [&](int k, double* tdst) {
      if (tid == 0) {
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        mbar_expect_tx(bar, piv_bytes + tab_bytes);
        bulk_g2s(B, piv + ((int64_t)k * Y4 + r0) * LD, piv_bytes, bar);
        bulk_g2s(tdst, tabc + Lt.stab + ((int64_t)k * Y + r0) * 8, tab_bytes, bar);
      }
    };
    issue_copies(steps - 1, sT[sc & 1]);

    // X-sweep unit of this warp: rows rg*32 + lane, columns [ib, ib + nx)
    const bool ax = warp < Ls.Ux;
    const int rg = ax ? warp / Ls.CHx : 0, chx = ax ? warp % Ls.CHx : 0;
    const int jl = rg * 32 + lane;
    const bool vr = ax && jl < Yc;
    const int ib = chx * K;
    const int nx = ax ? min(K, X - ib) : 0;
    const S* Arow = A + jl * LD;
    S* Brow = B + jl * LD;
    const S* uprow = nullptr;  // row above this lane's row, when lane 0 has to fetch it
    const S* dnrow = nullptr;  // row below, when it is not in the next lane
    if (vr && lane == 0) uprow = (jl > 0) ? A + (jl - 1) * LD : (Aprev ? Aprev + (Ycs - 1) * LD : nullptr);
    const bool dn_fetch = vr && (lane == 31 || jl == Yc - 1);
    if (dn_fetch) dnrow = (jl + 1 < Yc) ? A + (jl + 1) * LD : Anext;
    // Y-sweep unit of this warp: columns cgy*32 + lane, local rows [jb, jb + ny)
    const bool ay = warp < Ls.Uy;
    const int CHy = ceil_div(Yc, K);
    const int cgy = ay ? warp / Ls.CHy : 0, chy = ay ? warp % Ls.CHy : 0;
    const int col = cgy * 32 + lane;
    const bool vc = ay && col < X && chy < CHy;
    const int jb = chy * K;
    const int ny = (ay && chy < CHy) ? min(K, Yc - jb) : 0;

    // explicitY term of row jl at column i (:199); all lanes of the warp call it together
    auto vterm = [&](int i, S Rc, S g0, S g1, S g2) -> S {
      S up = __shfl_up_sync(FULL, Rc, 1);
      S dn = __shfl_down_sync(FULL, Rc, 1);
      if (lane == 0) up = uprow ? uprow[i] : (S)0;
      if (dn_fetch) dn = dnrow ? dnrow[i] : (S)0;
      return g0 * up + g1 * Rc + g2 * dn;
    };

    bool timed_out = false;  // a bulk-copy wait of this item gave up
    for (int s = 0; s < steps; s++, sc++) {
      const int k = steps - 1 - s;  // reverse (zip (init tl) (tail tl))  (:217)
      if (!mbar_wait(bar, phase, timed_out ? kWaitPollsAfterTimeout : kWaitPolls)) {
        timed_out = true;
        atomicExch(args.err, 3);
      }
      phase ^= 1u;
      if (clustered) cg::this_cluster().sync(); else __syncthreads();
      const double* tb = sT[sc & 1];
      const S dt = (S)tabc[Lt.dtinv + k];
      const S half = (S)0.5;
      const S e = vr ? (S)tb[jl * 8 + kSlotE] : (S)0;
      const S g0 = vr ? sG[4 * jl] : (S)0, g1 = vr ? sG[4 * jl + 1] : (S)0, g2 = vr ? sG[4 * jl + 2] : (S)0;

      // -------- X sweep pass 1: explicitX + explicitY, implicitX forward (chunk-local) --------
      S z[K];
      if (ax) {
        S zl = 0, Pl = 1;
        S Rl = (vr && ib > 0) ? Arow[ib - 1] : (S)0;
        S Rc = vr ? Arow[ib] : (S)0;
        S rbp = (vr && ib > 0) ? Brow[ib - 1] : (S)0;
#pragma unroll
        for (int m = 0; m < K; m++) {
          if (m < nx) {
            const int i = ib + m;
            const S Rn = (vr && i + 1 < X) ? Arow[i + 1] : (S)0;
            const S v = vterm(i, Rc, g0, g1, g2);
            const S aL = e * sW[i], aC = e * sW[Ls.xa + i], aR = e * sW[2 * Ls.xa + i];
            const S u = (dt + aC) * Rc + aL * Rl + aR * Rn + v;  // :195-200
            const S mult = aL * rbp;                             // -a_i / b'_{i-1}
            zl = u + mult * zl;
            Pl = mult * Pl;
            z[m] = zl;
            rbp = vr ? Brow[i] : (S)0;
            Rl = Rc;
            Rc = Rn;
          }
        }
        xfa[warp * 32 + lane] = zl;
        xfb[warp * 32 + lane] = Pl;
      }
      __syncthreads();
      // -------- pass 2: forward fix-up, backward recurrence (chunk-local) --------
      if (ax) {
        S zin = 0;
        for (int c2 = 0; c2 < chx; c2++) {
          const int u = rg * Ls.CHx + c2;
          zin = xfa[u * 32 + lane] + xfb[u * 32 + lane] * zin;
        }
        S P = 1;
        S rbp = (vr && ib > 0) ? Brow[ib - 1] : (S)0;
#pragma unroll
        for (int m = 0; m < K; m++) {
          if (m < nx) {
            const int i = ib + m;
            P = P * (e * sW[i] * rbp);
            z[m] = z[m] + P * zin;
            rbp = vr ? Brow[i] : (S)0;
          }
        }
        S xl = 0, Ql = 1;
#pragma unroll
        for (int m = K - 1; m >= 0; m--) {
          if (m < nx) {
            const int i = ib + m;
            const S rbm = vr ? Brow[i] : (S)0;
            const S nn = e * sW[2 * Ls.xa + i] * rbm;  // -c_i / b'_i
            xl = rbm * z[m] + nn * xl;
            Ql = nn * Ql;
            z[m] = xl;
          }
        }
        xba[warp * 32 + lane] = xl;
        xbb[warp * 32 + lane] = Ql;
      }
      __syncthreads();
      // -------- pass 3: backward fix-up, right-hand side of implicitY --------
      if (ax) {
        S xin = 0;
        for (int c2 = Ls.CHx - 1; c2 > chx; c2--) {
          const int u = rg * Ls.CHx + c2;
          xin = xba[u * 32 + lane] + xbb[u * 32 + lane] * xin;
        }
        S Q = 1;
#pragma unroll
        for (int m = K - 1; m >= 0; m--) {
          if (m < nx) {
            const int i = ib + m;
            const S rbm = vr ? Brow[i] : (S)0;
            Q = Q * (e * sW[2 * Ls.xa + i] * rbm);
            const S x = z[m] + Q * xin;
            const S Rc = vr ? Arow[i] : (S)0;
            const S v = vterm(i, Rc, g0, g1, g2);
            if (vr) Brow[i] = dt * x - half * v;  // dtInv * u - 0.5 * v  (:205)
          }
        }
      }
      __syncthreads();

      // -------- Y sweep: implicitY --------
      S y[K];
      S zz = 0;
      if (ny > 0) {
#pragma unroll
        for (int m = 0; m < K; m++) {
          if (m < ny) {
            const int j = jb + m;
            const S v = vc ? B[j * LD + col] : (S)0;
            zz = v + (S)tb[j * 8 + kSlotMY] * zz;
            y[m] = zz;
          }
        }
      }
      if (ay) yf[warp * 32 + lane] = zz;
      __syncthreads();
      // B is free again: bring in the next step's pivots and table
      if (s + 1 < steps) issue_copies(k - 1, sT[(sc + 1) & 1]);
      if (clustered) {
        for (int q = tid; q < Ls.CGy * 32; q += NT) {
          const int g = q >> 5, ln = q & 31;
          S a = 0;
          for (int c2 = 0; c2 < CHy; c2++) {
            const int je = min(Yc, c2 * K + K);
            a = yf[(g * Ls.CHy + c2) * 32 + ln] + (S)tb[(je - 1) * 8 + kSlotCP] * a;
          }
          blkF[q] = a;
        }
        if (tid == 0) {
          S b = 1;
          for (int c2 = 0; c2 < CHy; c2++) b = (S)tb[(min(Yc, c2 * K + K) - 1) * 8 + kSlotCP] * b;
          s_tot[0] = b;
        }
        cg::cluster_group cl = cg::this_cluster();
        cl.sync();
        for (int q = tid; q < Ls.CGy * 32; q += NT) {
          S zv = 0;
          for (int r = 0; r < rank; r++) {
            const S* rf = cl.map_shared_rank(blkF, r);
            const S* rt = cl.map_shared_rank(s_tot, r);
            zv = rf[q] + rt[0] * zv;
          }
          s_zin[q] = zv;
        }
        __syncthreads();
      }
      S xx = 0;
      if (ny > 0) {
        S zin = clustered ? s_zin[cgy * 32 + lane] : (S)0;
        for (int c2 = 0; c2 < chy; c2++)
          zin = yf[(cgy * Ls.CHy + c2) * 32 + lane] + (S)tb[(c2 * K + K - 1) * 8 + kSlotCP] * zin;
#pragma unroll
        for (int m = K - 1; m >= 0; m--) {
          if (m < ny) {
            const int j = jb + m;
            const S zv = y[m] + (S)tb[j * 8 + kSlotCP] * zin;
            xx = (S)tb[j * 8 + kSlotRB] * zv + (S)tb[j * 8 + kSlotNY] * xx;
            y[m] = xx;
          }
        }
      }
      if (ay) yb[warp * 32 + lane] = xx;
      __syncthreads();
      if (clustered) {
        for (int q = tid; q < Ls.CGy * 32; q += NT) {
          const int g = q >> 5, ln = q & 31;
          S a = 0;
          for (int c2 = CHy - 1; c2 >= 0; c2--) a = yb[(g * Ls.CHy + c2) * 32 + ln] + (S)tb[(c2 * K) * 8 + kSlotCQ] * a;
          blkB[q] = a;
        }
        if (tid == 0) {
          S b = 1;
          for (int c2 = CHy - 1; c2 >= 0; c2--) b = (S)tb[(c2 * K) * 8 + kSlotCQ] * b;
          s_tot[1] = b;
        }
        cg::cluster_group cl = cg::this_cluster();
        cl.sync();
        for (int q = tid; q < Ls.CGy * 32; q += NT) {
          S xv = 0;
          for (int r = C - 1; r > rank; r--) {
            const S* rb_ = cl.map_shared_rank(blkB, r);
            const S* rt = cl.map_shared_rank(s_tot, r);
            xv = rb_[q] + rt[1] * xv;
          }
          s_xin[q] = xv;
        }
        __syncthreads();
      }
      if (ny > 0) {
        S xin = clustered ? s_xin[cgy * 32 + lane] : (S)0;
        for (int c2 = CHy - 1; c2 > chy; c2--)
          xin = yb[(cgy * Ls.CHy + c2) * 32 + lane] + (S)tb[(c2 * K) * 8 + kSlotCQ] * xin;
#pragma unroll
        for (int m = 0; m < K; m++) {
          if (m < ny) {
            const int j = jb + m;
            const S xv = y[m] + (S)tb[j * 8 + kSlotCQ] * xin;
            if (vc) {
              A[j * LD + col] = xv;
              if (s == steps - 1 && col == c.xindex && r0 + j == c.yindex)
                args.out[c.out + item.strike] = (double)xv;  // myResult[myYindex, myXindex]
            }
          }
        }
      }
    }
  }
  // no CTA of a cluster may exit while a peer can still read its shared memory
  if (clustered) cg::this_cluster().sync();
}

}  // namespace lvc

namespace lvc {

// ---------------------------------------------------------------------------
// Full-tile line kernel: the same algorithm for grids whose line chunks, row
// groups and CTA row blocks are all full (numX % 32 == 0, rows per CTA a
// multiple of 32, numY divisible by the cluster size) -- every shape of the
// reference datasets and of the uneven calibration mix.  Each warp owns UPW
// units in each sweep (two independent recurrence chains per lane), which
// doubles the instruction-level parallelism and lets the register budget
// (up to 255 per thread with 8 warps) hold the chunk state without spilling.
// Without partial tiles there is no per-element predication; the grid buffer
// carries one halo row above and below (zero at the global boundary, written
// by the neighbouring CTA of the cluster during its Y sweep otherwise).
// ---------------------------------------------------------------------------
struct FullLayout {
  int LD, Ycs, CHx, Ux, CGy, CHy, Uy;
  int bar, A, B, wcol, grow, tab0, tab1, xfa, xfb, xba, xbb, yf, yb, blkF, blkB, zin, xin, tot, total;
};

template <typename S>
LVC_HD FullLayout full_layout(int X, int Ycs, int NU) {
  FullLayout L;
  auto up = [](int n) { return (n + 15) / 16 * 16; };
  const int s = (int)sizeof(S);
  L.LD = line_ld(X);
  L.Ycs = Ycs;
  L.CHx = X / kLineK;
  L.Ux = (Ycs / 32) * L.CHx;
  L.CGy = (X + 31) / 32;
  L.CHy = Ycs / kLineK;
  L.Uy = L.CGy * L.CHy;
  int o = 0;
  L.bar = o; o += 16;
  L.A = o; o += up((Ycs + 2) * L.LD * s);   // rows -1 .. Ycs (halo rows at both ends)
  L.B = o; o += up(Ycs * L.LD * s + 16);
  L.wcol = o; o += up(4 * X * s);           // [X][4]: W0, W1, W2, 0
  L.grow = o; o += up(4 * Ycs * s);
  L.tab0 = o; o += up(8 * Ycs * 8);
  L.tab1 = o; o += up(8 * Ycs * 8);
  L.xfa = o; o += up(NU * 32 * s);
  L.xfb = o; o += up(NU * 32 * s);
  L.xba = o; o += up(NU * 32 * s);
  L.xbb = o; o += up(NU * 32 * s);
  L.yf = o; o += up(NU * 32 * s);
  L.yb = o; o += up(NU * 32 * s);
  L.blkF = o; o += up(L.CGy * 32 * s);
  L.blkB = o; o += up(L.CGy * 32 * s);
  L.zin = o; o += up(L.CGy * 32 * s);
  L.xin = o; o += up(L.CGy * 32 * s);
  L.tot = o; o += up(4 * s);
  L.total = o;
  return L;
}

template <typename S> struct V2;
template <> struct V2<double> {
  static __device__ __forceinline__ double2 ld(const double* p) { return *reinterpret_cast<const double2*>(p); }
};
template <> struct V2<float> {
  static __device__ __forceinline__ float2 ld(const float* p) { return *reinterpret_cast<const float2*>(p); }
};

template <int NT> struct FullMinBlocks {
  static constexpr int v = NT >= 256 ? 1 : 256 / NT;
};

template <typename S, typename PV, int NT, int UPW>
__global__ void __launch_bounds__(NT, (FullMinBlocks<NT>::v)) lvc_line_full_kernel(RollbackArgs<S, PV> args) {
  constexpr int K = kLineK;
  constexpr int NW = NT / 32;
  constexpr int NU = NW * UPW;  // units per sweep
  static_assert(sizeof(S) == sizeof(PV), "pivots are copied verbatim into the state buffer");
  extern __shared__ __align__(16) unsigned char smem[];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int C = args.C;
  const bool clustered = C > 1;
  int rank = 0;
  if (clustered) rank = (int)cg::this_cluster().block_rank();
  const int cid = blockIdx.x / C, ncl = gridDim.x / C;
  unsigned sc = 0, phase = 0;
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem);
  if (tid == 0) {
    mbar_init(bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();

  for (int it = cid; it < args.n_items; it += ncl) {
    const Item item = args.items[it];
    const CalibDev c = args.calibs[item.calib];
    const int X = c.numX, Y = c.numY, T = c.numT;
    const int Ycs = c.Ycs;
    const int r0 = rank * Ycs;
    const FullLayout Ls = full_layout<S>(X, Ycs, NU);
    if (c.kind != kKindLine || c.C != C || c.ld != Ls.LD || Ls.total > args.smem_elems * (int)sizeof(S) ||
        Ls.Ux != NU || Ls.Uy != NU || (X % 32) || (Ycs % 32) || Ycs * C != Y) {
      if (tid == 0) atomicExch(args.err, 4);
      continue;
    }
    const int LD = Ls.LD;
    S* A = reinterpret_cast<S*>(smem + Ls.A);  // row r of the block at A + (r + 1) * LD
    S* B = reinterpret_cast<S*>(smem + Ls.B);
    const S* sW = reinterpret_cast<const S*>(smem + Ls.wcol);
    const S* sG = reinterpret_cast<const S*>(smem + Ls.grow);
    double* sT[2] = {reinterpret_cast<double*>(smem + Ls.tab0), reinterpret_cast<double*>(smem + Ls.tab1)};
    S* xfa = reinterpret_cast<S*>(smem + Ls.xfa);
    S* xfb = reinterpret_cast<S*>(smem + Ls.xfb);
    S* xba = reinterpret_cast<S*>(smem + Ls.xba);
    S* xbb = reinterpret_cast<S*>(smem + Ls.xbb);
    S* yf = reinterpret_cast<S*>(smem + Ls.yf);
    S* yb = reinterpret_cast<S*>(smem + Ls.yb);
    S* blkF = reinterpret_cast<S*>(smem + Ls.blkF);
    S* blkB = reinterpret_cast<S*>(smem + Ls.blkB);
    S* s_zin = reinterpret_cast<S*>(smem + Ls.zin);
    S* s_xin = reinterpret_cast<S*>(smem + Ls.xin);
    S* s_tot = reinterpret_cast<S*>(smem + Ls.tot);
    const double* tabc = args.tabs + c.tab;
    const TabLayout Lt = tab_layout(X, Y, T, c.Xp, kKindLine);
    const double strike = 0.001 * (double)item.strike;  // strikes (:247)
    const int steps = T > 1 ? T - 1 : 0;
    const PV* piv = args.piv + c.piv;
    const int64_t Y4 = round4(Y);
    S* halo_prev = nullptr;  // bottom halo row of rank - 1
    S* halo_next = nullptr;  // top halo row of rank + 1
    if (clustered) {
      cg::cluster_group cl = cg::this_cluster();
      if (rank > 0) halo_prev = cl.map_shared_rank(A + (Ycs + 1) * LD, rank - 1);
      if (rank < C - 1) halo_next = cl.map_shared_rank(A, rank + 1);
    }

    // The previous instance is done with every buffer, and -- across the
    // cluster -- every neighbour has finished pushing its last halo rows into
    // this CTA before they are re-initialised below.
    if (clustered) cg::this_cluster().sync(); else __syncthreads();
    // setPayoff (:46-47) on the block and on the halo rows (the payoff does not
    // depend on the row; halos at the global boundary are zero)
    for (int e = tid; e < (Ycs + 2) * LD; e += NT) {
      const int r = e / LD, i = e - r * LD;
      const bool boundary = (r == 0 && rank == 0) || (r == Ycs + 1 && rank == C - 1);
      A[e] = (i < X && !boundary) ? (S)fmax(tabc[Lt.x + i] - strike, 0.0) : (S)0;
    }
    for (int e = tid; e < 4 * X; e += NT) {
      const int i = e >> 2, k = e & 3;
      const_cast<S*>(sW)[e] = k < 3 ? (S)tabc[Lt.wcol + k * (int64_t)((X + 1) & ~1) + i] : (S)0;
    }
    for (int e = tid; e < 4 * Ycs; e += NT) const_cast<S*>(sG)[e] = (S)tabc[Lt.rowc + 4LL * r0 + e];

    if (steps == 0) {
      if (tid == 0 && c.yindex >= r0 && c.yindex < r0 + Ycs)
        args.out[c.out + item.strike] = fmax(tabc[Lt.x + c.xindex] - strike, 0.0);
      continue;
    }
    const unsigned piv_bytes = (unsigned)((Ycs * LD * (int)sizeof(S) + 15) & ~15);
    const unsigned tab_bytes = (unsigned)(Ycs * 64);
    auto issue_copies = [&](int k, double* tdst) {
      if (tid == 0) {
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        mbar_expect_tx(bar, piv_bytes + tab_bytes);
        bulk_g2s(B, piv + ((int64_t)k * Y4 + r0) * LD, piv_bytes, bar);
        bulk_g2s(tdst, tabc + Lt.stab + ((int64_t)k * Y + r0) * 8, tab_bytes, bar);
      }
    };
    issue_copies(steps - 1, sT[sc & 1]);

    // unit geometry (u = warp + slot * NW)
    int rgx[UPW], chx[UPW], jl[UPW], cgy[UPW], chy[UPW], colv[UPW];
#pragma unroll
    for (int q = 0; q < UPW; q++) {
      const int u = warp + q * NW;
      rgx[q] = u / Ls.CHx;
      chx[q] = u - rgx[q] * Ls.CHx;
      jl[q] = rgx[q] * 32 + lane;
      cgy[q] = u / Ls.CHy;
      chy[q] = u - cgy[q] * Ls.CHy;
      colv[q] = cgy[q] * 32 + lane;
    }
    // output lane: the unit and element holding myResult[myYindex, myXindex]
    int out_q = -1, out_m = 0;
#pragma unroll
    for (int q = 0; q < UPW; q++) {
      const int jy = c.yindex - r0 - chy[q] * K;
      if (colv[q] == c.xindex && jy >= 0 && jy < K) {
        out_q = q;
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
      if (clustered) cg::this_cluster().sync(); else __syncthreads();
      const double* tb = sT[sc & 1];
      const S dt = (S)tabc[Lt.dtinv + k];

      // -------- X sweep pass 1: explicitX + explicitY, forward recurrence (chunk-local) --------
      S z[UPW][K], PQ[UPW][K];
      {
        S e[UPW], g0[UPW], g1[UPW], g2[UPW], Rl[UPW], Rc[UPW], rbp[UPW], zl[UPW], Pl[UPW];
#pragma unroll
        for (int q = 0; q < UPW; q++) {
          const int ib = chx[q] * K;
          const S* Arow = A + (jl[q] + 1) * LD;
          e[q] = (S)tb[jl[q] * 8 + kSlotE];
          g0[q] = sG[4 * jl[q]];
          g1[q] = sG[4 * jl[q] + 1];
          g2[q] = sG[4 * jl[q] + 2];
          Rl[q] = ib > 0 ? Arow[ib - 1] : (S)0;
          Rc[q] = Arow[ib];
          rbp[q] = ib > 0 ? B[jl[q] * LD + ib - 1] : (S)0;
          zl[q] = 0;
          Pl[q] = 1;
        }
#pragma unroll
        for (int m = 0; m < K; m++) {
#pragma unroll
          for (int q = 0; q < UPW; q++) {
            const int i = chx[q] * K + m;
            const S* Arow = A + (jl[q] + 1) * LD;
            const S Rn = Arow[i + 1];  // column numX is zero padding
            const S up = Arow[i - LD];  // rows j-1 and j+1 (halo rows at the block edges)
            const S dn = Arow[i + LD];
            const auto w01 = V2<S>::ld(sW + 4 * i);
            const S w2 = sW[4 * i + 2];
            const S v = g0[q] * up + g1[q] * Rc[q] + g2[q] * dn;            // explicitY (:199)
            const S sx = w01.x * Rl[q] + w01.y * Rc[q] + w2 * Rn;           // explicitX / (0.5 e)
            const S u = e[q] * sx + (dt * Rc[q] + v);                       // :195-200
            const S mult = (e[q] * w01.x) * rbp[q];                         // -a_i / b'_{i-1}
            zl[q] = u + mult * zl[q];
            Pl[q] = mult * Pl[q];
            z[q][m] = zl[q];
            PQ[q][m] = Pl[q];
            rbp[q] = B[jl[q] * LD + i];
            Rl[q] = Rc[q];
            Rc[q] = Rn;
          }
        }
#pragma unroll
        for (int q = 0; q < UPW; q++) {
          const int u = warp + q * NW;
          xfa[u * 32 + lane] = zl[q];
          xfb[u * 32 + lane] = Pl[q];
        }
      }
      __syncthreads();
      // -------- pass 2: forward fix-up, backward recurrence (chunk-local) --------
      {
        S zin[UPW], xl[UPW], Ql[UPW], e[UPW];
#pragma unroll
        for (int q = 0; q < UPW; q++) {
          zin[q] = 0;
#pragma unroll 4
          for (int c2 = 0; c2 < chx[q]; c2++) {
            const int u = rgx[q] * Ls.CHx + c2;
            zin[q] = xfa[u * 32 + lane] + xfb[u * 32 + lane] * zin[q];
          }
          xl[q] = 0;
          Ql[q] = 1;
          e[q] = (S)tb[jl[q] * 8 + kSlotE];
        }
#pragma unroll
        for (int m = K - 1; m >= 0; m--) {
#pragma unroll
          for (int q = 0; q < UPW; q++) {
            const int i = chx[q] * K + m;
            const S zz = z[q][m] + PQ[q][m] * zin[q];
            const S rbm = B[jl[q] * LD + i];
            const S aR = e[q] * sW[4 * i + 2];
            xl[q] = rbm * (zz + aR * xl[q]);  // x_i = (z_i - c_i x_{i+1}) / b'_i
            Ql[q] = (aR * rbm) * Ql[q];
            z[q][m] = xl[q];
            PQ[q][m] = Ql[q];
          }
        }
#pragma unroll
        for (int q = 0; q < UPW; q++) {
          const int u = warp + q * NW;
          xba[u * 32 + lane] = xl[q];
          xbb[u * 32 + lane] = Ql[q];
        }
      }
      __syncthreads();
      // -------- pass 3: backward fix-up; dtInv * u goes to B (:205) --------
      {
        S xin[UPW];
#pragma unroll
        for (int q = 0; q < UPW; q++) {
          xin[q] = 0;
#pragma unroll 4
          for (int c2 = Ls.CHx - 1; c2 > chx[q]; c2--) {
            const int u = rgx[q] * Ls.CHx + c2;
            xin[q] = xba[u * 32 + lane] + xbb[u * 32 + lane] * xin[q];
          }
        }
#pragma unroll
        for (int m = 0; m < K; m++) {
#pragma unroll
          for (int q = 0; q < UPW; q++) {
            const int i = chx[q] * K + m;
            B[jl[q] * LD + i] = dt * (z[q][m] + PQ[q][m] * xin[q]);
          }
        }
      }
      __syncthreads();

      // -------- Y sweep --------
      S y[UPW][K];
      {
        S zz[UPW], Ru[UPW], Rm[UPW];
#pragma unroll
        for (int q = 0; q < UPW; q++) {
          zz[q] = 0;
          const int j0 = chy[q] * K;
          Ru[q] = A[j0 * LD + colv[q]];        // row j0 - 1 (halo row at the block edge)
          Rm[q] = A[(j0 + 1) * LD + colv[q]];  // row j0
        }
#pragma unroll
        for (int m = 0; m < K; m++) {
#pragma unroll
          for (int q = 0; q < UPW; q++) {
            const int j = chy[q] * K + m;
            const S Rd = A[(j + 2) * LD + colv[q]];  // row j + 1
            const auto g01 = V2<S>::ld(sG + 4 * j);
            const S v = g01.x * Ru[q] + g01.y * Rm[q] + sG[4 * j + 2] * Rd;  // explicitY (:199)
            const S rhs = B[j * LD + colv[q]] - (S)0.5 * v;                   // :205
            zz[q] = rhs + (S)tb[j * 8 + kSlotMY] * zz[q];
            y[q][m] = zz[q];
            Ru[q] = Rm[q];
            Rm[q] = Rd;
          }
        }
#pragma unroll
        for (int q = 0; q < UPW; q++) yf[(warp + q * NW) * 32 + lane] = zz[q];
      }
      __syncthreads();
      if (s + 1 < steps) issue_copies(k - 1, sT[(sc + 1) & 1]);
      if (clustered) {
        for (int qq = tid; qq < Ls.CGy * 32; qq += NT) {
          const int g = qq >> 5, ln = qq & 31;
          S a = 0;
          for (int c2 = 0; c2 < Ls.CHy; c2++) a = yf[(g * Ls.CHy + c2) * 32 + ln] + (S)tb[(c2 * K + K - 1) * 8 + kSlotCP] * a;
          blkF[qq] = a;
        }
        if (tid == 0) {
          S b = 1;
          for (int c2 = 0; c2 < Ls.CHy; c2++) b = (S)tb[(c2 * K + K - 1) * 8 + kSlotCP] * b;
          s_tot[0] = b;
        }
        cg::cluster_group cl = cg::this_cluster();
        cl.sync();
        for (int qq = tid; qq < Ls.CGy * 32; qq += NT) {
          S zv = 0;
          for (int r = 0; r < rank; r++) {
            const S* rf = cl.map_shared_rank(blkF, r);
            const S* rt = cl.map_shared_rank(s_tot, r);
            zv = rf[qq] + rt[0] * zv;
          }
          s_zin[qq] = zv;
        }
        __syncthreads();
      }
      {
        S zin[UPW], xx[UPW];
#pragma unroll
        for (int q = 0; q < UPW; q++) {
          zin[q] = clustered ? s_zin[cgy[q] * 32 + lane] : (S)0;
#pragma unroll 4
          for (int c2 = 0; c2 < chy[q]; c2++)
            zin[q] = yf[(cgy[q] * Ls.CHy + c2) * 32 + lane] + (S)tb[(c2 * K + K - 1) * 8 + kSlotCP] * zin[q];
          xx[q] = 0;
        }
#pragma unroll
        for (int m = K - 1; m >= 0; m--) {
#pragma unroll
          for (int q = 0; q < UPW; q++) {
            const int j = chy[q] * K + m;
            const double2 nr = *reinterpret_cast<const double2*>(tb + j * 8 + kSlotNY);  // nY, 1/b'
            const S zv = y[q][m] + (S)tb[j * 8 + kSlotCP] * zin[q];
            xx[q] = (S)nr.y * zv + (S)nr.x * xx[q];
            y[q][m] = xx[q];
          }
        }
#pragma unroll
        for (int q = 0; q < UPW; q++) yb[(warp + q * NW) * 32 + lane] = xx[q];
      }
      __syncthreads();
      if (clustered) {
        for (int qq = tid; qq < Ls.CGy * 32; qq += NT) {
          const int g = qq >> 5, ln = qq & 31;
          S a = 0;
          for (int c2 = Ls.CHy - 1; c2 >= 0; c2--) a = yb[(g * Ls.CHy + c2) * 32 + ln] + (S)tb[(c2 * K) * 8 + kSlotCQ] * a;
          blkB[qq] = a;
        }
        if (tid == 0) {
          S b = 1;
          for (int c2 = Ls.CHy - 1; c2 >= 0; c2--) b = (S)tb[(c2 * K) * 8 + kSlotCQ] * b;
          s_tot[1] = b;
        }
        cg::cluster_group cl = cg::this_cluster();
        cl.sync();
        for (int qq = tid; qq < Ls.CGy * 32; qq += NT) {
          S xv = 0;
          for (int r = C - 1; r > rank; r--) {
            const S* rb_ = cl.map_shared_rank(blkB, r);
            const S* rt = cl.map_shared_rank(s_tot, r);
            xv = rb_[qq] + rt[1] * xv;
          }
          s_xin[qq] = xv;
        }
        __syncthreads();
      }
      {
        S xin[UPW];
#pragma unroll
        for (int q = 0; q < UPW; q++) {
          xin[q] = clustered ? s_xin[cgy[q] * 32 + lane] : (S)0;
#pragma unroll 4
          for (int c2 = Ls.CHy - 1; c2 > chy[q]; c2--)
            xin[q] = yb[(cgy[q] * Ls.CHy + c2) * 32 + lane] + (S)tb[(c2 * K) * 8 + kSlotCQ] * xin[q];
        }
#pragma unroll
        for (int m = 0; m < K; m++) {
#pragma unroll
          for (int q = 0; q < UPW; q++) {
            const int j = chy[q] * K + m;
            const S xv = y[q][m] + (S)tb[j * 8 + kSlotCQ] * xin[q];
            y[q][m] = xv;
            A[(j + 1) * LD + colv[q]] = xv;
          }
        }
        // halo rows of the cluster neighbours, and the price on the last step
#pragma unroll
        for (int q = 0; q < UPW; q++) {
          if (halo_prev && chy[q] == 0) halo_prev[colv[q]] = y[q][0];
          if (halo_next && chy[q] == Ls.CHy - 1) halo_next[colv[q]] = y[q][K - 1];
        }
        if (s == steps - 1 && out_q >= 0) {
          S pv = 0;
#pragma unroll
          for (int q = 0; q < UPW; q++)
#pragma unroll
            for (int m = 0; m < K; m++)
              if (q == out_q && m == out_m) pv = y[q][m];
          args.out[c.out + item.strike] = (double)pv;  // myResult[myYindex, myXindex]
        }
      }
    }
  }
  if (clustered) cg::this_cluster().sync();
}

}  // namespace lvc
