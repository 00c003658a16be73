// The turbulent-kinetic-energy step of the ocean model,
// misc/ocean-sim/tke.fut (entry main, DTYPE = f32), behind the C API the
// Futhark compiler generates for that program (include/tke.h).  A library of
// its own: the program's entry point is named futhark_entry_main like
// LocVolCalib's.
//
// One step is three kernels: tke_column_kernel on the context's stream and
// tke_advect_kernel on an auxiliary stream run side by side (the first is
// latency-bound, the second issue-bound, and they share no data), then
// tke_ab_kernel applies the Adams-Bashforth update (:341-347) once both are
// done.
//   tke_advect_kernel  the advection fluxes east, north and top
//                      (tke.fut:264-319) and dtketau (:320-340).  A thread
//                      owns one (y, z) of a (y, z) tile of the plane and
//                      marches along x over a segment, carrying the east flux
//                      of x - 1 in a register; the north flux of y - 1 and the
//                      top flux of z - 1 come from the neighbouring threads
//                      through shared memory, so each flux is evaluated about
//                      once.
//   tke_column_kernel  everything else, one lane per (x, y) column, a warp per
//                      32 consecutive columns: the coefficients (:103-210) and
//                      tridagPar's two forward recurrences
//                      (misc/ocean-sim/tridiag.fut:9-56) in one pass down the
//                      column, the backward recurrence (:61-79), the water
//                      mask, the surface correction, clip and lateral
//                      diffusion of the top cell (:212-263), giving tketaup1
//                      before the Adams-Bashforth update.  The four fields
//                      the coefficients need are staged through shared
//                      memory in chunks of 4 z
//                      (cp.async, three stages) as [z][column] tiles, so both
//                      the coalesced copy and the lane-per-column reads are
//                      free of bank conflicts; the forward pass leaves the two
//                      quotients of the backward recurrence, y'/b' and -c/b',
//                      in an L2-resident [z][column] scratch.
// Every operation is explicitly rounded (no fused multiply-add) in the
// reference's operand order -- the fold order of each recurrence included --
// so the outputs equal the CPU oracle's, which reproduces the reference's
// golden outputs, bit for bit.  Quotients by a divisor that stays fixed over
// many of them (dz of a level, cos * dy of a row, cos * dx of a step) come
// from its double reciprocal (DR_), which gives the same correctly rounded
// float as the division.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <string>

#include "tke.h"
#include "fut_api.cuh"

namespace {

__device__ __forceinline__ float M_(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float A_(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float S_(float a, float b) { return __fsub_rn(a, b); }
// a / b correctly rounded.  A zero dividend over a finite non-zero divisor is
// answered directly (IEEE 754: a zero whose sign is the XOR of the operands'
// signs): such quotients are common here -- dry cells have a = c = d = 0 --
// and would otherwise leave the division's fast path.
__device__ __forceinline__ float D_(float a, float b) {
  if (a == 0.0f && b != 0.0f && fabsf(b) <= 3.402823466e38f)
    return __int_as_float((__float_as_int(a) ^ __float_as_int(b)) & (int)0x80000000);
  return __fdiv_rn(a, b);
}
// a / b correctly rounded, from rb = 1 / (double)b correctly rounded in
// double (Rd_): the float nearest the double product a * rb.  That product
// is within 2^-52 of a / b relatively, while a quotient of two floats (24-bit
// significands A, B) is never a point halfway between two floats and never
// closer to one than 2^-49 relatively (a nonzero multiple of a power of two
// over B < 2^24, against a result below 2^25 of the same power): the product
// therefore rounds to float as a / b does -- the argument that makes double
// rounding harmless when the wider format carries at least 2p + 2 bits.
// Zeros and infinities and the signs follow from the IEEE operations
// (0 * rb = +-0, a * inf for b = 0).  One double reciprocal then serves every
// quotient with that divisor, each at the cost of one double multiply and
// two conversions.
__device__ __forceinline__ double Rd_(float b) { return __drcp_rn((double)b); }
__device__ __forceinline__ float DR_(float a, double rb) { return __double2float_rn(__dmul_rn((double)a, rb)); }
// std::max / std::min as the oracle evaluates them
__device__ __forceinline__ float max_(float a, float b) { return (a < b) ? b : a; }
__device__ __forceinline__ float min_(float a, float b) { return (b < a) ? b : a; }

constexpr float kDtTracer = 1.0f, kDtTke = 1.0f, kAlphaTke = 1.0f, kCEps = 0.7f, kKhTke = 2000.0f, kABEps = 0.1f;

struct TkeArgs {
  int X, Y, Z;
  const float *tketau, *tketaup1, *dtketau, *dtketaum1, *utau, *vtau, *wtau, *maskU, *maskV, *maskW;
  const float *dxt, *dxu, *dyt, *dyu, *dzt, *dzw, *cost, *cosu;
  const int32_t* kbot;
  const float *kappaM, *mxl, *forc, *forc_tke_surface;
  float *q0, *q1;         // scratch [zdim][ncolp]: y'_z / b'_z and -c_z / b'_z of each column
  int64_t ncolp;          // xdim * ydim rounded up to 32
  float *tketaup1_out, *dtketau_out, *tke_surf_corr_out;  // outputs
};

__device__ __forceinline__ int64_t i3(const TkeArgs& p, int x, int y, int z) {
  return ((int64_t)x * p.Y + y) * p.Z + z;
}
__device__ __forceinline__ bool interior(const TkeArgs& p, int x, int y) {
  return x >= 2 && x < p.X - 2 && y >= 2 && y < p.Y - 2;
}

// tke.fut:19-41
__device__ __forceinline__ float limiter(float cr) {
  return max_(0.0f, max_(min_(1.0f, M_(2.0f, cr)), min_(2.0f, cr)));
}
// uCFL is |scaledVel dt_tracer / dx|: from dx itself (RECIP false) or from
// its double reciprocal rdx (RECIP true, DR_)
template <bool RECIP>
__device__ __forceinline__ float calcflux(float velfac, float velS, float dt_tracer, float dx, double rdx,
                                          float varS, float varSM1, float varSP1, float varSP2, float maskS,
                                          float maskSM1, float maskSP1) {
  const float scaledVel = M_(velfac, velS);
  const float uCFL = fabsf(RECIP ? DR_(M_(scaledVel, dt_tracer), rdx) : D_(M_(scaledVel, dt_tracer), dx));
  const float rjp = M_(S_(varSP2, varSP1), maskSP1);
  const float rj = M_(S_(varSP1, varS), maskS);
  const float rjm = M_(S_(varS, varSM1), maskSM1);
  const float epsilon = 0.00000000000000000001f;
  const float divisor = (fabsf(rj) < epsilon) ? epsilon : rj;
  float cr = D_((velS > 0.0f) ? rjm : rjp, divisor);  // one division of the selected dividend
  cr = limiter(cr);
  return S_(M_(M_(scaledVel, A_(varSP1, varS)), 0.5f),
            M_(M_(M_(fabsf(scaledVel), A_(S_(1.0f, cr), M_(uCFL, cr))), rj), 0.5f));
}

// lateral diffusion fluxes (:236-251), from tketau
__device__ __forceinline__ float diff_east(const TkeArgs& p, int x, int y, int z) {
  if (!(x < p.X - 1)) return 0.0f;
  const int64_t i = i3(p, x, y, z);
  return M_(D_(M_(kKhTke, S_(p.tketau[i3(p, x + 1, y, z)], p.tketau[i])), M_(p.cost[y], p.dxu[x])), p.maskU[i]);
}
__device__ __forceinline__ float diff_north(const TkeArgs& p, int x, int y, int z) {
  if (!(y < p.Y - 1)) return 0.0f;
  const int64_t i = i3(p, x, y, z);
  return M_(M_(D_(M_(kKhTke, S_(p.tketau[i3(p, x, y + 1, z)], p.tketau[i])), p.dyu[y]), p.maskV[i]), p.cosu[y]);
}
// advection fluxes (:264-319)
__device__ __forceinline__ float adv_east(const TkeArgs& p, int x, int y, int z) {
  if (!(x >= 1 && x < p.X - 2 && y >= 2 && y < p.Y - 2)) return 0.0f;
  const int64_t i = i3(p, x, y, z);
  const float dx = M_(p.cost[y], p.dxt[x]);
  const float mWm1 = p.maskW[i3(p, x - 1, y, z)], mWs = p.maskW[i], mWp1 = p.maskW[i3(p, x + 1, y, z)],
              mWp2 = p.maskW[i3(p, x + 2, y, z)];
  const bool in = x < p.X - 1;
  return calcflux<false>(1.0f, p.utau[i], kDtTracer, dx, 0.0, p.tketau[i], p.tketau[i3(p, x - 1, y, z)],
                  p.tketau[i3(p, x + 1, y, z)], p.tketau[i3(p, x + 2, y, z)], in ? M_(mWs, mWp1) : 0.0f,
                  in ? M_(mWm1, mWs) : 0.0f, in ? M_(mWp1, mWp2) : 0.0f);
}
// ---------------------------------------------------------------------------
// tke_advect_kernel
// ---------------------------------------------------------------------------
constexpr int kAdvThreads = 256;  // at <= 64 registers two CTAs fit beside two column-kernel CTAs

// Block b.x covers a tile of ty rows (y) x tz levels (z) of the plane -- the
// halo row 0 in warp 0, row r >= 1 at threads 32 + (r - 1) tz .., z fastest,
// the z extent split into nzt tiles of at most 31 owned levels, level 0 of a
// tile being halo too -- and block b.y the x segment
// [b.y * xseg, ...).  A thread keeps tketau and maskW of x - 1 .. x + 2 at
// its (y, z) in registers (the east flux, :264-281) and publishes those of x
// in shared memory, where its neighbours (y +- 1, y + 2) and (z +- 1, z + 2)
// read them for the north (:282-299) and top (:300-319) fluxes -- from
// global memory where the neighbour is outside the tile.  The north flux of
// (y - 1, z) is thread t - tz's and the top flux of (y, z - 1) thread
// t - 1's, again through shared memory, for every owned cell: the halo row
// and level compute those fluxes in the same code as everyone else.  Tiles
// (rather than runs of consecutive (y, z)) keep most north neighbours in the
// block when zdim is large: with zdim = 100, 2.56 rows of 256 threads held
// none of them.
__global__ void __launch_bounds__(kAdvThreads, 4) tke_advect_kernel(TkeArgs p, int xseg, int ty, int tz, int nzt) {
  __shared__ float sT[kAdvThreads], sW[kAdvThreads], sfn[kAdvThreads], sft[kAdvThreads];
  const int t = threadIdx.x;
  const int64_t plane = (int64_t)p.Y * p.Z;
  const int Z = p.Z;
  // position in the tile: the halo row in warp 0 (lanes 0 .. tz - 1), rows
  // 1 .. ty - 1 packed from thread 32 on, so the halo row's warp evaluates
  // only the north flux the row above needs
  const bool hwarp = t < 32;
  const int ry = hwarp ? 0 : 1 + (t - 32) / tz, rz = hwarp ? t : (t - 32) % tz;
  const int yt = blockIdx.x / nzt, zt = blockIdx.x - yt * nzt;
  // row 0 and level 0 of the tile are halo: the cells just below the owned
  // (ty - 1) x (tz - 1) ones, whose north and top fluxes the owned cells
  // need; they run the same flux code, so no warp evaluates a neighbour's
  // flux on a divergent path
  const int yy = yt * (ty - 1) + ry - 1, zz = zt * (tz - 1) + rz - 1;
  const bool live = ry < ty && rz < tz && yy >= 0 && yy < p.Y && zz >= 0 && zz < Z;
  const bool owned = live && ry >= 1 && rz >= 1;
  const int y = live ? yy : 0, z = live ? zz : 0;
  const int64_t qi = (int64_t)y * Z + z;
  const int xs = blockIdx.y * xseg, xe = min(p.X, xs + xseg);
  const bool n_in = ry >= 1 && ry + 2 < ty;  // (y - 1 .. y + 2, z) in this tile
  const int nm = ry == 1 ? t - 32 : t - tz, np1 = hwarp ? t + 32 : t + tz;  // threads of rows y - 1, y + 1
  const bool t_in = rz >= 1 && rz + 2 < tz;  // (y, z - 1 .. z + 2) in this tile
  const bool yint = y >= 2 && y < p.Y - 2;
  const float cy = live ? p.cost[y] : 1.0f, cuy = live ? p.cosu[y] : 1.0f, dyt = live ? p.dyt[y] : 1.0f;
  const float dz = live ? p.dzw[z] : 1.0f;
  // the divisors that stay fixed along x, as double reciprocals (DR_)
  const double rdy = Rd_(M_(cy, dyt)), rdz = Rd_(dz), rhdz = Rd_(M_(0.5f, dz));
  auto ldT = [&](int xx) { return (live && xx >= 0 && xx < p.X) ? p.tketau[xx * plane + qi] : 0.0f; };
  auto ldW = [&](int xx) { return (live && xx >= 0 && xx < p.X) ? p.maskW[xx * plane + qi] : 0.0f; };
  float T0 = ldT(xs - 1), T1 = ldT(xs), T2 = ldT(xs + 1), T3 = ldT(xs + 2);  // x - 1 .. x + 2
  float W0 = ldW(xs - 1), W1 = ldW(xs), W2 = ldW(xs + 1), W3 = ldW(xs + 2);
  float fe_prev = (live && !hwarp && xs >= 1) ? adv_east(p, xs - 1, y, z) : 0.0f;
  // the velocities of this thread's cell, one step ahead
  auto ldU = [&](const float* f, int xx) { return (live && xx < xe) ? f[xx * plane + qi] : 0.0f; };
  float uN = ldU(p.utau, xs), vN = ldU(p.vtau, xs), wN = ldU(p.wtau, xs);
  for (int x = xs; x < xe; x++) {
    const int64_t i = x * plane + qi;
    sT[t] = T1;
    sW[t] = W1;
    const float nT = ldT(x + 3), nW = ldW(x + 3);  // next step's window end
    const float uC = uN, vC = vN, wC = wN;
    uN = ldU(p.utau, x + 1);
    vN = ldU(p.vtau, x + 1);
    wN = ldU(p.wtau, x + 1);
    __syncthreads();
    float fe = 0.0f, fn = 0.0f, ft = 0.0f;
    const double rdx = Rd_(M_(cy, p.dxt[x]));  // the east divisor of this x, for fe and dtketau
    if (live) {
      const bool xint = x >= 2 && x < p.X - 2;
      if (!hwarp && x >= 1 && x < p.X - 2 && yint) {
        const bool in = x < p.X - 1;
        fe = calcflux<true>(1.0f, uC, kDtTracer, 0.0f, rdx, T1, T0, T2, T3, in ? M_(W1, W2) : 0.0f,
                      in ? M_(W0, W1) : 0.0f, in ? M_(W2, W3) : 0.0f);
      }
      if (y >= 1 && y < p.Y - 2 && xint) {
        float tm, tp1, tp2, wm, wp1, wp2;
        if (n_in) {
          tm = sT[nm];
          tp1 = sT[np1];
          tp2 = sT[np1 + tz];
          wm = sW[nm];
          wp1 = sW[np1];
          wp2 = sW[np1 + tz];
        } else {
          tm = p.tketau[i - Z];
          tp1 = p.tketau[i + Z];
          tp2 = p.tketau[i + 2 * Z];
          wm = p.maskW[i - Z];
          wp1 = p.maskW[i + Z];
          wp2 = p.maskW[i + 2 * Z];
        }
        const bool in = y < p.Y - 1;
        fn = calcflux<true>(cuy, vC, kDtTracer, 0.0f, rdy, T1, tm, tp1, tp2, in ? M_(W1, wp1) : 0.0f,
                      in ? M_(wm, W1) : 0.0f, in ? M_(wp1, wp2) : 0.0f);
      }
      if (!hwarp && z < Z - 1 && xint && yint) {
        float tm = 0.0f, tp1, tp2 = 0.0f, wm = 0.0f, wp1, wp2 = 0.0f;
        if (t_in) {
          if (z != 0) {
            tm = sT[t - 1];
            wm = sW[t - 1];
          }
          tp1 = sT[t + 1];
          wp1 = sW[t + 1];
          if (z < Z - 2) {
            tp2 = sT[t + 2];
            wp2 = sW[t + 2];
          }
        } else {
          if (z != 0) {
            tm = p.tketau[i - 1];
            wm = p.maskW[i - 1];
          }
          tp1 = p.tketau[i + 1];
          wp1 = p.maskW[i + 1];
          if (z < Z - 2) {
            tp2 = p.tketau[i + 2];
            wp2 = p.maskW[i + 2];
          }
        }
        ft = calcflux<true>(1.0f, wC, kDtTracer, 0.0f, rdz, T1, tm, tp1, tp2, M_(W1, wp1), M_(wm, W1), M_(wp1, wp2));
      }
    }
    sfn[t] = fn;
    sft[t] = ft;
    __syncthreads();
    if (owned) {  // dtketau (:320-340)
      const float fnm = sfn[nm];  // the north flux of (y - 1, z): 0 outside the domain
      const float ftm = sft[t - 1];   // the top flux of (y, z - 1)
      float tmp;
      if (x >= 2 && x < p.X - 2 && yint)
        tmp = M_(W1, S_(DR_(-S_(fe, fe_prev), rdx), DR_(S_(fn, fnm), rdy)));
      else
        tmp = p.dtketau[i];
      const float z0 = z == 0 ? S_(tmp, DR_(ft, rdz)) : tmp;
      const float zm = (z >= 1 && z < Z - 1) ? S_(z0, DR_(S_(ft, ftm), rdz)) : z0;
      p.dtketau_out[i] = (z == Z - 1) ? S_(zm, DR_(S_(ft, ftm), rhdz)) : zm;
    }
    fe_prev = fe;
    T0 = T1;
    T1 = T2;
    T2 = T3;
    T3 = nT;
    W0 = W1;
    W1 = W2;
    W2 = W3;
    W3 = nW;
  }
}

// ---------------------------------------------------------------------------
// tke_column_kernel
// ---------------------------------------------------------------------------
constexpr int kColWarps = 4;   // warps per CTA, each on its own 32 columns
constexpr int kColCh = 4;      // z values per staged chunk (a power of two <= 32)
constexpr int kColStages = 3;  // chunks in flight: current, next (kappaM[z + 1]), prefetch
constexpr int kColPad = 33;    // [z][column] tile row stride
constexpr int kColStageFloats = 4 * kColCh * kColPad;  // tketau, kappaM, mxl, forc
constexpr int kColWarpFloats = kColStages * kColStageFloats + kColCh * kColPad;  // + output tile
constexpr size_t kColSmem = sizeof(float) * kColWarps * kColWarpFloats;

__device__ __forceinline__ void cp_async4(float* dst, const float* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all_but_one() {
  asm volatile("cp.async.wait_group 1;\n" ::: "memory");
}

// Chunk k (z = k*kColCh .. +kColCh-1) of the four fields of columns
// col0 .. col0+31 into st[field][z - k*kColCh][column]: lane l copies
// z = k*kColCh + l % kColCh of columns l / kColCh + j * (32 / kColCh), so a
// warp instruction reads runs of kColCh floats of 32 / kColCh columns.
__device__ __forceinline__ void col_stage_chunk(const TkeArgs& p, float* st, int64_t col0, int64_t ncol, int k,
                                                int lane) {
  const int zz = lane & (kColCh - 1), z = k * kColCh + zz;
  if (z >= p.Z) return;
#pragma unroll
  for (int j = 0; j < kColCh; j++) {
    const int c = j * (32 / kColCh) + lane / kColCh;
    const int64_t col = col0 + c;
    if (col < ncol) {
      const int64_t g = col * p.Z + z;
      float* d = st + zz * kColPad + c;
      cp_async4(d, p.tketau + g);
      cp_async4(d + kColCh * kColPad, p.kappaM + g);
      cp_async4(d + 2 * kColCh * kColPad, p.mxl + g);
      cp_async4(d + 3 * kColCh * kColPad, p.forc + g);
    }
  }
}

// Chunk k of tketaup1 -- what a cell keeps where the solution does not apply
// -- into st[z - k*kColCh][column], in the pattern of col_stage_chunk.
constexpr int kColUpdFloats = kColCh * kColPad;
static_assert(2 * kColUpdFloats <= kColStages * kColStageFloats, "update stages reuse the forward stages");
__device__ __forceinline__ void col_stage_update(const TkeArgs& p, float* st, int64_t col0, int64_t ncol, int k,
                                                 int lane) {
  const int zz = lane & (kColCh - 1), z = k * kColCh + zz;
  if (z >= p.Z) return;
#pragma unroll
  for (int j = 0; j < kColCh; j++) {
    const int c = j * (32 / kColCh) + lane / kColCh;
    const int64_t col = col0 + c;
    if (col < ncol) {
      const int64_t g = col * p.Z + z;
      float* d = st + zz * kColPad + c;
      cp_async4(d, p.tketaup1 + g);
    }
  }
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// At most 128 registers (four CTAs' worth per SM): two CTAs then leave room
// for two advection CTAs beside them.
__global__ void __launch_bounds__(kColWarps * 32, 4) tke_column_kernel(TkeArgs p) {
  extern __shared__ float smem[];
  constexpr unsigned kAll = 0xffffffffu;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t ncol = (int64_t)p.X * p.Y;
  const int64_t col0 = ((int64_t)blockIdx.x * kColWarps + warp) * 32;
  if (col0 >= ncol) return;  // whole warps only; the warps of a CTA share no barrier
  float* st = smem + warp * kColWarpFloats;
  float* tile = st + kColStages * kColStageFloats;
  const int Z = p.Z;
  const int64_t col = col0 + lane;
  const bool valid = col < ncol;
  const int x = valid ? (int)(col / p.Y) : 0, y = valid ? (int)(col % p.Y) : 0;
  const bool inner = valid && interior(p, x, y);
  const int ks = valid ? p.kbot[col] - 1 : -1;
  const bool land = ks >= 0;
  const float fts = inner ? p.forc_tke_surface[col] : 0.0f;
  const int nch = (Z + kColCh - 1) / kColCh;
  const int64_t qs = p.ncolp;
  float* q0 = p.q0 + col;
  float* q1 = p.q1 + col;

  // Forward, staged a chunk of kColCh z at a time and computed one z at a
  // time (a rolled loop: the unrolled chunk body cost more than its overlap
  // of the coefficients of neighbouring z saved): (A) the coefficients
  // (tke.fut:103-210); (B) tridagPar's recurrences 1 (the 4-tuple scan for
  // b', tridiag.fut:9-33) and 2 (y', :38-56) folded left to right --
  // recurrence 2 at z needs b' of z - 1 only; (C) the two quotients the
  // backward recurrence folds.  Every lane runs A and B (the shuffles need
  // the whole warp); only interior columns store.
  float s0 = 1.0f, s1 = 0.0f, s2 = 0.0f, s3 = 1.0f, b0 = 0.0f, y0 = 0.0f, r0 = 0.0f, r1 = 1.0f;
  float dm = 0.0f, cprev = 0.0f;
  double rbpprev = 0.0;  // 1 / b' of z - 1 (DR_)
  col_stage_chunk(p, st, col0, ncol, 0, lane);
  cp_async_commit();
  if (nch > 1) col_stage_chunk(p, st + kColStageFloats, col0, ncol, 1, lane);
  cp_async_commit();
  // the per-z constants of the next chunk, loaded a chunk ahead: lane l
  // holds dzw and dzt of z + 1 for z = (chunk) * kColCh + l % kColCh
  float dzN = 1.0f, dztN = 1.0f;
  auto ld_consts = [&](int k) {
    const int zl = k * kColCh + (lane & (kColCh - 1));
    dzN = zl < Z ? p.dzw[zl] : 1.0f;
    dztN = zl < Z - 1 ? p.dzt[zl + 1] : 1.0f;
  };
  ld_consts(0);
  for (int k = 0; k < nch; k++) {
    if (k + 2 < nch) col_stage_chunk(p, st + ((k + 2) % kColStages) * kColStageFloats, col0, ncol, k + 2, lane);
    cp_async_commit();
    cp_async_wait_all_but_one();  // chunks k and k + 1 have landed
    __syncwarp();
    const float* cur = st + (k % kColStages) * kColStageFloats;
    const float* nxt = st + ((k + 1) % kColStages) * kColStageFloats;
    const int zbase = k * kColCh;
    const int zn = min(kColCh, Z - zbase);
    // the chunk's per-z constants, lane l holding those of z = zbase + l % kColCh
    const float dz_l = dzN;
    const float fac_l = zbase + (lane & (kColCh - 1)) < Z - 1 ? M_(M_(D_(kDtTke, dztN), kAlphaTke), 0.5f) : 0.0f;
    const double rdz_l = Rd_(dz_l);  // the quotients by dz of the interior levels (DR_)
    if (k + 1 < nch) ld_consts(k + 1);
#pragma unroll 1
    for (int zz = 0; zz < zn; zz++) {  // (A), (B), (C) for one z
      const float fac = __shfl_sync(kAll, fac_l, zz);
      const float dz = __shfl_sync(kAll, dz_l, zz);
      const double rdz = __shfl_sync(kAll, rdz_l, zz);
      const int z = zbase + zz;
      const float t = cur[zz * kColPad + lane];
      const float kap = cur[(kColCh + zz) * kColPad + lane];
      const float mx = cur[(2 * kColCh + zz) * kColPad + lane];
      const float fo = cur[(3 * kColCh + zz) * kColPad + lane];
      const float kapn = zz + 1 < kColCh ? cur[(kColCh + zz + 1) * kColPad + lane] : nxt[kColCh * kColPad + lane];
      const float d0 = z < Z - 1 ? M_(fac, A_(kap, kapn)) : 0.0f;  // delta (:103-108)
      const bool edge = land && z == ks, water = land && z >= ks;
      const float sq = __fsqrt_rn(max_(0.0f, t));
      float a_ = 0.0f, b_ = 0.0f, c_ = 0.0f, d_ = 0.0f;
      if (edge || !water) a_ = 0.0f;
      else if (z > 0 && z < Z - 1) a_ = DR_(-dm, rdz);
      else if (z == Z - 1) a_ = D_(-dm, M_(0.5f, dz));
      if (!water) b_ = 1.0f;
      else if (edge) b_ = A_(A_(1.0f, DR_(d0, rdz)), M_(__fdiv_rn(M_(kDtTke, kCEps), mx), sq));
      else if (z > 0 && z < Z - 1) b_ = A_(A_(1.0f, DR_(A_(d0, dm), rdz)), __fdiv_rn(M_(M_(kDtTke, kCEps), sq), mx));
      else if (z == Z - 1) b_ = A_(A_(1.0f, D_(dm, M_(0.5f, dz))), M_(D_(M_(kDtTke, kCEps), mx), sq));
      if (z < Z - 1) c_ = water ? DR_(-d0, rdz) : 0.0f;
      if (water) {
        const float tmp = A_(t, M_(kDtTke, fo));
        d_ = (z == Z - 1) ? A_(tmp, D_(M_(kDtTke, fts), M_(0.5f, dz))) : tmp;
      }
      dm = d0;
      float m0 = 1.0f, m1 = 0.0f, m2 = 0.0f, m3 = 1.0f;
      if (z > 0) {
        m0 = b_;
        m1 = S_(0.0f, M_(a_, cprev));
        m2 = 1.0f;
        m3 = 0.0f;
      } else {
        b0 = b_;
      }
      const float value = __frcp_rn(M_(s0, m0));
      const float n0 = M_(A_(M_(m0, s0), M_(m1, s2)), value);
      const float n1 = M_(A_(M_(m0, s1), M_(m1, s3)), value);
      const float n2 = M_(A_(M_(m2, s0), M_(m3, s2)), value);
      const float n3 = M_(A_(M_(m2, s1), M_(m3, s3)), value);
      s0 = n0;
      s1 = n1;
      s2 = n2;
      s3 = n3;
      // (quotients whose dividend is rarely zero skip D_'s test for one)
      const float bpz = __fdiv_rn(A_(M_(s0, b0), s1), A_(M_(s2, b0), s3));
      const double rbp = Rd_(bpz);  // three quotients by b'_z: y'_z, c_z here, a_{z+1} next
      float l0 = 0.0f, l1 = 1.0f;
      if (z > 0) {
        l0 = d_;
        l1 = S_(0.0f, DR_(a_, rbpprev));
      } else {
        y0 = d_;
      }
      const float rn0 = A_(l0, M_(l1, r0)), rn1 = M_(r1, l1);
      r0 = rn0;
      r1 = rn1;
      const float ypz = A_(r0, M_(r1, y0));
      cprev = c_;
      rbpprev = rbp;
      if (inner) {
        const int64_t o = (int64_t)z * qs;
        q0[o] = DR_(ypz, rbp);
        q1[o] = S_(0.0f, DR_(c_, rbp));
      }
    }
    __syncwarp();  // the next iteration refills this chunk's stage
  }
  cp_async_wait_all();

  // Backward, a chunk at a time from the top: recurrence 3 down the column
  // into the tile, then the chunk's cells (coalesced): take the solution or
  // keep tketaup1 (:212-218), the top cell's correction, clip and lateral
  // diffusion (:219-263) -- tketaup1 before the Adams-Bashforth update, which
  // tke_ab_kernel applies once the advection kernel is done.  The quotients
  // of the chunk after next (registers) and tketaup1 three chunks on
  // (cp.async) load meanwhile: a backward chunk is little work, so one chunk
  // ahead left the loads' latency exposed.
  float* ust = st;
  const float yn = inner ? q0[(int64_t)(Z - 1) * qs] : 0.0f;  // y'_{n-1} / b'_{n-1}
  r0 = 0.0f;
  r1 = 1.0f;
  if (valid && !inner) p.tke_surf_corr_out[col] = 0.0f;
  // quotients of chunk k (qa), k - 1 (qb) and k - 2 (loaded this iteration)
  // in registers; tketaup1 of chunks k .. k - kUpd + 1 in flight (cp.async)
  constexpr int kUpd = 4;
  static_assert(kUpd * kColUpdFloats <= kColStages * kColStageFloats, "update stages reuse the forward stages");
  auto ldq = [&](int k, float (&d0)[kColCh], float (&d1)[kColCh]) {  // element n - 1 folds the neutral (0, 1)
#pragma unroll
    for (int zz = 0; zz < kColCh; zz++) {
      const int z = k * kColCh + zz;
      const bool ld = inner && k >= 0 && z < Z - 1;
      d0[zz] = ld ? q0[(int64_t)z * qs] : 0.0f;
      d1[zz] = ld ? q1[(int64_t)z * qs] : 1.0f;
    }
  };
  float qa0[kColCh], qa1[kColCh], qb0[kColCh], qb1[kColCh];
  ldq(nch - 1, qa0, qa1);
  ldq(nch - 2, qb0, qb1);
  for (int d = 0; d < kUpd - 1; d++) {
    if (nch - 1 - d >= 0) col_stage_update(p, ust + ((nch - 1 - d) % kUpd) * kColUpdFloats, col0, ncol, nch - 1 - d, lane);
    cp_async_commit();
  }
  int in_c[kColCh], ks_c[kColCh];  // the flags of the columns this lane stores
#pragma unroll
  for (int j = 0; j < kColCh; j++) {
    const int c = j * (32 / kColCh) + lane / kColCh;
    in_c[j] = __shfl_sync(kAll, (int)inner, c);
    ks_c[j] = __shfl_sync(kAll, ks, c);
  }
  for (int k = nch - 1; k >= 0; k--) {
    const int zn = min(kColCh, Z - k * kColCh);
    float qc0[kColCh], qc1[kColCh];
    if (k - (kUpd - 1) >= 0)
      col_stage_update(p, ust + ((k - (kUpd - 1)) % kUpd) * kColUpdFloats, col0, ncol, k - (kUpd - 1), lane);
    cp_async_commit();
    ldq(k - 2, qc0, qc1);
    if (inner) {
#pragma unroll
      for (int zz = kColCh - 1; zz >= 0; zz--) {
        if (zz >= zn) continue;
        const int z = k * kColCh + zz;
        const float rn0 = A_(qa0[zz], M_(qa1[zz], r0)), rn1 = M_(r1, qa1[zz]);
        r0 = rn0;
        r1 = rn1;
        float v = A_(r0, M_(r1, yn));
        if (z == Z - 1) {  // the top cell
          float tp = (land && z >= ks) ? v : p.tketaup1[col * Z + z];
          p.tke_surf_corr_out[col] = tp < 0.0f ? D_(M_(M_(-tp, 0.5f), p.dzw[Z - 1]), kDtTke) : 0.0f;
          tp = tp < 0.0f ? 0.0f : tp;
          v = A_(tp, M_(M_(kDtTke, p.maskW[col * Z + z]),
                        A_(D_(S_(diff_east(p, x, y, z), diff_east(p, x - 1, y, z)), M_(p.cost[y], p.dxt[x])),
                           D_(S_(diff_north(p, x, y, z), diff_north(p, x, y - 1, z)), M_(p.cost[y], p.dyt[y])))));
        }
        tile[zz * kColPad + lane] = v;
      }
    }
    asm volatile("cp.async.wait_group %0;\n" ::"n"(kUpd - 1) : "memory");  // chunk k's update fields have landed
    __syncwarp();
    const float* u = ust + (k % kUpd) * kColUpdFloats;
#pragma unroll
    for (int j = 0; j < kColCh; j++) {
      const int c = j * (32 / kColCh) + lane / kColCh, zz = lane & (kColCh - 1);
      const int64_t cc = col0 + c;
      if (cc < ncol && zz < zn) {
        const int z = k * kColCh + zz;
        const bool take = in_c[j] && (z == Z - 1 || (ks_c[j] >= 0 && z >= ks_c[j]));
        const float* uf = u + zz * kColPad + c;
        p.tketaup1_out[cc * Z + z] = take ? tile[zz * kColPad + c] : uf[0];
      }
    }
    __syncwarp();  // the tile and this stage are rewritten by later chunks
#pragma unroll
    for (int zz = 0; zz < kColCh; zz++) {
      qa0[zz] = qb0[zz];
      qa1[zz] = qb1[zz];
      qb0[zz] = qc0[zz];
      qb1[zz] = qc1[zz];
    }
  }
}

// Adams-Bashforth (tke.fut:341-347) on the column kernel's tketaup1, with
// dtketau from the advection kernel: both have finished when it runs.
__device__ __forceinline__ float ab_update(float tp1, float dt, float dtm1) {
  return A_(tp1, M_(kDtTracer, S_(M_(A_(1.5f, kABEps), dt), M_(A_(0.5f, kABEps), dtm1))));
}
// Four cells per thread and access (16-byte loads and stores) where the three
// arrays allow it, the rest one at a time.
__global__ void __launch_bounds__(256) tke_ab_kernel(TkeArgs p) {
  const int64_t n = (int64_t)p.X * p.Y * p.Z;
  const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x, nth = (int64_t)gridDim.x * blockDim.x;
  const bool vec = ((reinterpret_cast<uintptr_t>(p.tketaup1_out) | reinterpret_cast<uintptr_t>(p.dtketau_out) |
                     reinterpret_cast<uintptr_t>(p.dtketaum1)) & 15) == 0;
  int64_t i0 = 0;
  if (vec) {
    const int64_t n4 = n / 4;
    float4* tp = reinterpret_cast<float4*>(p.tketaup1_out);
    const float4* dt = reinterpret_cast<const float4*>(p.dtketau_out);
    const float4* dm = reinterpret_cast<const float4*>(p.dtketaum1);
    for (int64_t j = tid; j < n4; j += nth) {
      const float4 a = tp[j], b = dt[j], c = __ldcs(dm + j);
      __stcs(tp + j, make_float4(ab_update(a.x, b.x, c.x), ab_update(a.y, b.y, c.y), ab_update(a.z, b.z, c.z),
                                 ab_update(a.w, b.w, c.w)));
    }
    i0 = 4 * n4;
  }
  for (int64_t i = i0 + tid; i < n; i += nth)
    p.tketaup1_out[i] = ab_update(p.tketaup1_out[i], p.dtketau_out[i], p.dtketaum1[i]);
}

int64_t padded_columns(int64_t X, int64_t Y) { return (X * Y + 31) & ~int64_t(31); }

size_t scratch_bytes(int64_t X, int64_t Y, int64_t Z) {
  // the two quotient planes q0, q1 of [zdim][ncolp] floats
  return 2 * sizeof(float) * (size_t)std::max<int64_t>(32, Z * padded_columns(X, Y));
}

// Enqueues one step on the context's stream (lock held, device set).
int step_launch(futhark_context* ctx, const tke_step_args* q) {
  const int64_t X = q->xdim, Y = q->ydim, Z = q->zdim;
  if (X < 0 || Y < 0 || Z < 0 || X > INT32_MAX || Y > INT32_MAX || Z > INT32_MAX)
    return set_error(ctx, FUTHARK_PROGRAM_ERROR, "tke step: bad array dimensions");
  // the reference's dtketau reads flux_top[x, y, zdim - 2] at z = zdim - 1
  // (tke.fut:338): index -1, a bounds failure, when zdim is 1
  if (Z == 1 && X * Y > 0)
    return set_error(ctx, FUTHARK_PROGRAM_ERROR, "tke step: index [-1] out of bounds for zdim 1 (tke.fut:338)");
  const int64_t n = X * Y * Z;
  if (n == 0) return 0;
  if (((uintptr_t)q->scratch & 127) != 0)
    return set_error(ctx, FUTHARK_PROGRAM_ERROR, "tke step: scratch is not on a 128-byte boundary");
  float* scratch = static_cast<float*>(q->scratch);
  TkeArgs p;
  p.X = (int)X;
  p.Y = (int)Y;
  p.Z = (int)Z;
  p.tketau = q->tketau;
  p.tketaup1 = q->tketaup1;
  p.dtketau = q->dtketau;
  p.dtketaum1 = q->dtketaum1;
  p.utau = q->utau;
  p.vtau = q->vtau;
  p.wtau = q->wtau;
  p.maskU = q->maskU;
  p.maskV = q->maskV;
  p.maskW = q->maskW;
  p.dxt = q->dxt;
  p.dxu = q->dxu;
  p.dyt = q->dyt;
  p.dyu = q->dyu;
  p.dzt = q->dzt;
  p.dzw = q->dzw;
  p.cost = q->cost;
  p.cosu = q->cosu;
  p.kbot = q->kbot;
  p.kappaM = q->kappaM;
  p.mxl = q->mxl;
  p.forc = q->forc;
  p.forc_tke_surface = q->forc_tke_surface;
  p.ncolp = padded_columns(X, Y);
  p.q0 = scratch;
  p.q1 = scratch + Z * p.ncolp;
  p.tketaup1_out = q->tketaup1_out;
  p.dtketau_out = q->dtketau_out;
  p.tke_surf_corr_out = q->tke_surf_corr_out;
  cudaStream_t s = ctx->stream;
  if (!ensure_aux_stream(ctx)) return set_error(ctx, FUTHARK_PROGRAM_ERROR, "tke step: cannot create a stream");
  // The column kernel (latency-bound, a warp per 32 columns) on the context's
  // stream and the advection kernel (issue-bound) on the auxiliary stream run
  // side by side: they share no data until tke_ab_kernel.
  cudaError_t e = cudaEventRecord(ctx->ev_fork, s);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(ctx->aux, ctx->ev_fork, 0);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "tke step fork");
  // the columns: coefficients, tridagPar, tketaup1 (tke.fut:103-263)
  const int64_t col_blocks = (X * Y + 32 * kColWarps - 1) / (32 * kColWarps);
  if (col_blocks > INT32_MAX) return set_error(ctx, FUTHARK_PROGRAM_ERROR, "tke step: too many columns");
  if (!ctx->smem_raised) {  // once per context: host time the step need not spend
    e = cudaFuncSetAttribute((const void*)tke_column_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)kColSmem);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "tke column attributes");
    ctx->smem_raised = true;
  }
  tke_column_kernel<<<(unsigned)col_blocks, 32 * kColWarps, kColSmem, s>>>(p);
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(ctx, e, "tke column launch");
  // advection and dtketau: (y, z) tiles of at most 31 owned levels plus a
  // halo level and a halo row, x segments so that about four waves of CTAs run
  const int64_t nzt = (Z + 30) / 31, tz = (Z + nzt - 1) / nzt + 1, ty = 1 + (kAdvThreads - 32) / tz;
  const int64_t plane_blocks = ((Y + ty - 2) / (ty - 1)) * nzt;
  const int64_t want_blocks = 4LL * 4 * ctx->num_sms;  // four CTAs per SM
  const int64_t nseg = std::max<int64_t>(1, std::min<int64_t>(X, (want_blocks + plane_blocks - 1) / plane_blocks));
  const int xseg = (int)((X + nseg - 1) / nseg);
  const int64_t segs = (X + xseg - 1) / xseg;
  if (plane_blocks > INT32_MAX || segs > 65535)
    return set_error(ctx, FUTHARK_PROGRAM_ERROR, "tke step: plane too large");
  tke_advect_kernel<<<dim3((unsigned)plane_blocks, (unsigned)segs), kAdvThreads, 0, ctx->aux>>>(p, xseg, (int)ty,
                                                                                                (int)tz, (int)nzt);
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(ctx, e, "tke advection launch");
  e = cudaEventRecord(ctx->ev_join, ctx->aux);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(s, ctx->ev_join, 0);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "tke step join");
  // Adams-Bashforth (:341-347)
  tke_ab_kernel<<<(unsigned)std::min<int64_t>((n + 255) / 256, 8LL * ctx->num_sms), 256, 0, s>>>(p);
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(ctx, e, "tke update launch");
  return 0;
}

// Synchronises the context's stream and reports a failed step (lock held).
int check_locked(futhark_context* ctx) {
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  if (e == cudaSuccess) e = cudaGetLastError();
  return e == cudaSuccess ? 0 : cuda_fail(ctx, e, "tke step");
}

}  // namespace

extern "C" {
FUT_ARRAY_API(f32_1d, float, 1, int64_t dim0)
FUT_ARRAY_API(f32_2d, float, 2, int64_t dim0, int64_t dim1)
FUT_ARRAY_API(f32_3d, float, 3, int64_t dim0, int64_t dim1, int64_t dim2)
FUT_ARRAY_API(i32_2d, int32_t, 2, int64_t dim0, int64_t dim1)

int futhark_entry_main(struct futhark_context* ctx, struct futhark_f32_3d** out0, struct futhark_f32_3d** out1,
                       struct futhark_f32_3d** out2, struct futhark_f32_3d** out3, struct futhark_f32_3d** out4,
                       struct futhark_f32_3d** out5, struct futhark_f32_2d** out6, struct futhark_f32_3d* tketau,
                       struct futhark_f32_3d* tketaup1, struct futhark_f32_3d* tketaum1,
                       struct futhark_f32_3d* dtketau, struct futhark_f32_3d* dtketaup1,
                       struct futhark_f32_3d* dtketaum1, const struct futhark_f32_3d* utau,
                       const struct futhark_f32_3d* vtau, const struct futhark_f32_3d* wtau,
                       const struct futhark_f32_3d* maskU, const struct futhark_f32_3d* maskV,
                       const struct futhark_f32_3d* maskW, const struct futhark_f32_1d* dxt,
                       const struct futhark_f32_1d* dxu, const struct futhark_f32_1d* dyt,
                       const struct futhark_f32_1d* dyu, const struct futhark_f32_1d* dzt,
                       const struct futhark_f32_1d* dzw, const struct futhark_f32_1d* cost,
                       const struct futhark_f32_1d* cosu, const struct futhark_i32_2d* kbot,
                       const struct futhark_f32_3d* kappaM, const struct futhark_f32_3d* mxl,
                       const struct futhark_f32_3d* forc, const struct futhark_f32_2d* forc_tke_surface) {
  std::lock_guard<std::mutex> g(ctx->mu);
  if (!ctx->ok) return set_error(ctx, FUTHARK_PROGRAM_ERROR, "context has no usable CUDA device");
  if (!out0 || !out1 || !out2 || !out3 || !out4 || !out5 || !out6)
    return set_error(ctx, FUTHARK_PROGRAM_ERROR, "null output pointer");
  const futhark_f32_3d* a3[] = {tketau, tketaup1, tketaum1, dtketau, dtketaup1, dtketaum1, utau, vtau,
                                wtau,   maskU,    maskV,    maskW,   kappaM,    mxl,       forc};
  for (auto* v : a3)
    if (!v) return set_error(ctx, FUTHARK_PROGRAM_ERROR, "null array");
  const int64_t X = tketau->shape[0], Y = tketau->shape[1], Z = tketau->shape[2];
  for (auto* v : a3)
    if (v->shape[0] != X || v->shape[1] != Y || v->shape[2] != Z)
      return set_error(ctx, FUTHARK_PROGRAM_ERROR, "tke main: the [xdim][ydim][zdim] inputs differ in shape");
  auto need1 = [&](const futhark_f32_1d* v, int64_t len) { return v && v->shape[0] == len; };
  if (!need1(dxt, X) || !need1(dxu, X) || !need1(dyt, Y) || !need1(dyu, Y) || !need1(dzt, Z) || !need1(dzw, Z) ||
      !need1(cost, Y) || !need1(cosu, Y) || !kbot || kbot->shape[0] != X || kbot->shape[1] != Y ||
      !forc_tke_surface || forc_tke_surface->shape[0] != X || forc_tke_surface->shape[1] != Y)
    return set_error(ctx, FUTHARK_PROGRAM_ERROR, "tke main: an input's size does not match xdim, ydim or zdim");
  if (X > INT32_MAX || Y > INT32_MAX || Z > INT32_MAX)
    return set_error(ctx, FUTHARK_PROGRAM_ERROR, "tke main: array dimension too large");
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "tke main");
  const int64_t d3[3] = {X, Y, Z}, d2[2] = {X, Y};
  futhark_f32_3d* up1 = alloc_array<futhark_f32_3d>(d3, 3);
  futhark_f32_3d* dtk = alloc_array<futhark_f32_3d>(d3, 3);
  futhark_f32_2d* corr = alloc_array<futhark_f32_2d>(d2, 2);
  if (!up1 || !dtk || !corr || !ensure_scratch(ctx, scratch_bytes(X, Y, Z))) {
    drop_array(up1);
    drop_array(dtk);
    drop_array(corr);
    return set_error(ctx, FUTHARK_OUT_OF_MEMORY, "out of device memory");
  }
  tke_step_args q;
  q.xdim = X;
  q.ydim = Y;
  q.zdim = Z;
  q.tketau = tketau->data;
  q.tketaup1 = tketaup1->data;
  q.dtketau = dtketau->data;
  q.dtketaum1 = dtketaum1->data;
  q.utau = utau->data;
  q.vtau = vtau->data;
  q.wtau = wtau->data;
  q.maskU = maskU->data;
  q.maskV = maskV->data;
  q.maskW = maskW->data;
  q.dxt = dxt->data;
  q.dxu = dxu->data;
  q.dyt = dyt->data;
  q.dyu = dyu->data;
  q.dzt = dzt->data;
  q.dzw = dzw->data;
  q.cost = cost->data;
  q.cosu = cosu->data;
  q.kbot = kbot->data;
  q.kappaM = kappaM->data;
  q.mxl = mxl->data;
  q.forc = forc->data;
  q.forc_tke_surface = forc_tke_surface->data;
  q.tketaup1_out = up1->data;
  q.dtketau_out = dtk->data;
  q.tke_surf_corr_out = corr->data;
  q.scratch = ctx->scratch;
  int rc = step_launch(ctx, &q);
  if (!rc) rc = check_locked(ctx);
  // the four state arrays the step returns unchanged (tke.fut:348)
  futhark_f32_3d* pass[4] = {};
  const futhark_f32_3d* src[4] = {tketau, tketaum1, dtketaup1, dtketaum1};
  for (int k = 0; k < 4 && !rc; k++) {
    pass[k] = new (std::nothrow) futhark_f32_3d(*src[k]);
    if (!pass[k]) rc = set_error(ctx, FUTHARK_OUT_OF_MEMORY, "out of host memory");
    else pass[k]->mem->refs++;
  }
  if (rc) {
    for (auto* v : pass) drop_array(v);
    drop_array(up1);
    drop_array(dtk);
    drop_array(corr);
    return rc;
  }
  *out0 = pass[0];
  *out1 = up1;
  *out2 = pass[1];
  *out3 = dtk;
  *out4 = pass[2];
  *out5 = pass[3];
  *out6 = corr;
  return 0;
}

size_t tke_scratch_bytes(int64_t xdim, int64_t ydim, int64_t zdim) {
  if (xdim < 0 || ydim < 0 || zdim < 0) return 0;
  return scratch_bytes(xdim, ydim, zdim);
}
int tke_step_f32(struct futhark_context* ctx, const struct tke_step_args* args) {
  std::lock_guard<std::mutex> g(ctx->mu);
  if (!ctx->ok) return set_error(ctx, FUTHARK_PROGRAM_ERROR, "context has no usable CUDA device");
  if (!args) return set_error(ctx, FUTHARK_PROGRAM_ERROR, "null step arguments");
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "tke step");
  return step_launch(ctx, args);
}
int tke_check(struct futhark_context* ctx) {
  std::lock_guard<std::mutex> g(ctx->mu);
  if (!ctx->ok) return set_error(ctx, FUTHARK_PROGRAM_ERROR, "context has no usable CUDA device");
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "tke check");
  return check_locked(ctx);
}
void* tke_context_stream(struct futhark_context* ctx) { return ctx && ctx->ok ? (void*)ctx->stream : nullptr; }
int tke_launches_per_step(void) { return 3; }

}  // extern "C"
