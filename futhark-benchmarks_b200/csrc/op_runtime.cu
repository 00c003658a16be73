// finpar/OptionPricing.fut (entry main, f32) behind the C API the Futhark
// compiler generates for it (include/op.h): Sobol quasi-random paths through
// an inverse Gaussian, a Brownian bridge and a Black-Scholes model, priced
// under one of three contracts and averaged per model.
//
// op_paths_kernel<C> is specialised on the contract C, which fixes a path's
// shape (dates x underlyings: contract 1 is 1 x 1, contract 2 is 5 x 3,
// contract 3 is 367 x 3, the reference's size coercions at :294-298), so
// every loop over a path has a constant trip count and the paths of contracts
// 1 and 2 stay in registers.  A thread prices a contiguous range of paths:
// the first path's Sobol point is assembled from the set bits of its Gray
// code (:13-33); each following path n differs from n - 1 in one Gray-code
// bit, so its point is the previous one XOR one direction vector per
// dimension.  The Gaussians are computed on the fly inside the Brownian
// bridge recursion, the correlated prices date by date with a running
// product (the scan of :217), and the payoff is decided as the dates go by,
// so a path holds only its Sobol integers and the bridge values.  Each
// thread accumulates its payoffs per model in f64, each CTA adds its threads'
// sums in a fixed tree order, and op_reduce_kernel adds the CTAs' sums, again
// in a fixed order, and divides by num_mc_it in f32.
//
// Arithmetic: this file is compiled with --fmad=false, so every f32
// operation is rounded on its own as in the reference (and the CPU oracle);
// division and square root are IEEE; f32.exp and f32.log are the f32
// rounding of CUDA's f64 exp and log.  The kernel is compute-bound (about
// 1e5 operations per path of contract 3, mostly the inverse Gaussian and the
// exponentials).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <string>
#include <vector>

#include "op.h"
#include "fut_api.cuh"

namespace {

template <int C>
struct OpShape;
// kMinCtas: the thread-per-path kernel's CTAs per SM the register budget is
// sized for (contract 2's 15-dimension paths want the registers of one)
template <>
struct OpShape<1> {
  static constexpr int D = 1, U = 1, kMinCtas = 4;
};
template <>
struct OpShape<2> {
  static constexpr int D = 5, U = 3, kMinCtas = 3;
};
template <>
struct OpShape<3> {  // priced by op_paths_warp_kernel
  static constexpr int D = 367, U = 3;
};

constexpr int kOpThreads = 128;  // thread-per-path CTAs: contract 2 fits three per SM
constexpr int kOpModels = 4;  // models priced per launch (accumulators in registers)

struct OpDev {
  int num_mc_it, num_bits, num_models, num_discts;
  const int32_t* dir_vs;
  const float *md_cs, *md_vols, *md_drifts, *md_sts, *md_detvals, *md_discts;
  const int32_t* bb_inds;
  const float* bb_data;
  float* pay_out;  // reference order: every path's payoff, [path][model]; null otherwise
};

__device__ __forceinline__ float f32exp(float x) { return (float)exp((double)x); }
__device__ __forceinline__ float f32log(float x) { return (float)log((double)x); }

// Wichura's AS241 coefficient tables (:59-118), as the reference's f32 literals
__constant__ float kSmallA[8] = {3.387132872796366608f, 133.14166789178437745f, 1971.5909503065514427f,
                                 13731.693765509461125f, 45921.953931549871457f, 67265.770927008700853f,
                                 33430.575583588128105f, 2509.0809287301226727f};
__constant__ float kSmallB[8] = {1.0f, 42.313330701600911252f, 687.1870074920579083f, 5394.1960214247511077f,
                                 21213.794301586595867f, 39307.89580009271061f, 28729.085735721942674f,
                                 5226.495278852854561f};
__constant__ float kInterA[8] = {1.42343711074968357734f, 4.6303378461565452959f, 5.7694972214606914055f,
                                 3.64784832476320460504f, 1.27045825245236838258f, 0.24178072517745061177f,
                                 0.0227238449892691845833f, 7.7454501427834140764e-4f};
__constant__ float kInterB[8] = {1.0f, 2.05319162663775882187f, 1.6763848301838038494f, 0.68976733498510000455f,
                                 0.14810397642748007459f, 0.0151986665636164571966f, 5.475938084995344946e-4f,
                                 1.05075007164441684324e-9f};
__constant__ float kTailA[8] = {6.6579046435011037772f, 5.4637849111641143699f, 1.7848265399172913358f,
                                0.29656057182850489123f, 0.026532189526576123093f, 0.0012426609473880784386f,
                                2.71155556874348757815e-5f, 2.01033439929228813265e-7f};
__constant__ float kTailB[8] = {1.0f, 0.59983220655588793769f, 0.13692988092273580531f, 0.0148753612908506148525f,
                                7.868691311456132591e-4f, 1.8463183175100546818e-5f, 1.4215117583164458887e-7f,
                                2.04426310338993978564e-5f};

// :52-57
__device__ __forceinline__ float poly_appr(float x, const float* a, const float* b) {
  const float num = x * (x * (x * (x * (x * (x * (x * a[7] + a[6]) + a[5]) + a[4]) + a[3]) + a[2]) + a[1]) + a[0];
  const float den = x * (x * (x * (x * (x * (x * (x * b[7] + b[6]) + b[5]) + b[4]) + b[3]) + b[2]) + b[1]) + b[0];
  return num / den;
}

// :120-136, split at its branch: gauss_central for |p - 0.5| <= 0.425,
// gauss_tail otherwise
__device__ __forceinline__ bool gauss_is_central(float dp) {
  return (dp < 0.0f && 0.0f - dp <= 0.425f) || (0.0f <= dp && dp <= 0.425f);
}
__device__ __forceinline__ float gauss_central(float dp) {
  return dp * poly_appr(0.180625f - dp * dp, kSmallA, kSmallB);
}
__device__ __forceinline__ float gauss_tail(float dp) {
  const float pp = dp < 0.0f ? dp + 0.5f : 0.5f - dp;
  const float r = sqrtf(-f32log(pp));
  const float x = r <= 5.0f ? poly_appr(r - 1.6f, kInterA, kInterB) : poly_appr(r - 5.0f, kTailA, kTailB);
  return dp < 0.0f ? 0.0f - x : x;
}
__device__ __forceinline__ float ugaussian_el(float p) {
  const float dp = p - 0.5f;
  return gauss_is_central(dp) ? gauss_central(dp) : gauss_tail(dp);
}

// :234-240
__device__ __forceinline__ float fmin_payoff(const float* xs) {
  const float a = xs[0] / 3758.05f, b = xs[1] / 11840.0f, c = xs[2] / 1200.0f;
  return a < b ? (a < c ? a : c) : (b < c ? b : c);
}

// bb_inds selects dates of the path: bi[0] always, and from i = 1 on
// bi[i], ri[i] in 1 .. D and li[i] in 0 .. D (0: no left point).  Kernels
// that find otherwise price nothing and return NaN instead of reading
// outside the path (the entry point rejects such inputs before launching).
template <int D>
__device__ bool bridge_indices_valid(const int32_t* ind) {
  bool ok = ind[0] >= 1 && ind[0] <= D;
  for (int i = 1; i < D; i++)
    ok = ok && ind[i] >= 1 && ind[i] <= D && ind[D + i] >= 0 && ind[D + i] <= D && ind[2 * D + i] >= 1 &&
         ind[2 * D + i] <= D;
  return ok;
}

template <int C>
__global__ void __launch_bounds__(kOpThreads, OpShape<C>::kMinCtas) op_paths_kernel(OpDev a, int m0, double* __restrict__ partial) {
  constexpr int D = OpShape<C>::D, U = OpShape<C>::U, K = D * U;
  __shared__ int32_t s_ind[3 * D];  // bb_inds: bi, li, ri
  __shared__ float s_dat[3 * D];    // bb_data: sd, lw, rw
  __shared__ int s_ok;
  for (int i = threadIdx.x; i < 3 * D; i += blockDim.x) {
    s_ind[i] = a.bb_inds[i];
    s_dat[i] = a.bb_data[i];
  }
  __syncthreads();
  if (threadIdx.x == 0) s_ok = bridge_indices_valid<D>(s_ind);
  __syncthreads();
  const bool ok = s_ok;
  const int64_t T = (int64_t)gridDim.x * blockDim.x;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t N = ok ? a.num_mc_it : 0;
  const int64_t lo = N * t / T, hi = N * (t + 1) / T;
  const int B = a.num_bits;
  const uint32_t bits = B >= 32 ? 0xffffffffu : ((1u << B) - 1u);
  const float divisor = ldexpf(1.0f, B);  // 2 ** num_bits, exact
  const int nm = min(kOpModels, a.num_models - m0);
  double acc[kOpModels];
#pragma unroll
  for (int mm = 0; mm < kOpModels; mm++) acc[mm] = 0.0;
  int32_t xs[K];  // the path's Sobol integers, dimension k = date * U + underlying
  float bb[K];    // the Brownian bridge, [date][underlying]
  for (int64_t it = lo; it < hi; it++) {
    const int32_t n = (int32_t)(it + 1);
    if (it == lo) {  // from the Gray code's set bits (:13-33)
      for (int k = 0; k < K; k++) xs[k] = 0;
      for (uint32_t g = (uint32_t)((n >> 1) ^ n) & bits; g != 0u; g &= g - 1u) {
        const int i = __ffs((int)g) - 1;
        for (int k = 0; k < K; k++) xs[k] ^= a.dir_vs[(int64_t)k * B + i];
      }
    } else {  // Gray code of n = that of n - 1 with bit ctz(n) flipped
      const int c = __ffs(n) - 1;
      if (c < B)
        for (int k = 0; k < K; k++) xs[k] ^= a.dir_vs[(int64_t)k * B + c];
    }
    // Brownian bridge per underlying (:142-175), Gaussians on the fly
    for (int k = 0; k < K; k++) bb[k] = 0.0f;
    for (int u = 0; u < U; u++) {
      bb[(s_ind[0] - 1) * U + u] = s_dat[0] * ugaussian_el((float)xs[u] / divisor);
      for (int i = 1; i < D; i++) {
        const int j = s_ind[D + i] - 1, kk = s_ind[2 * D + i] - 1, l = s_ind[i] - 1;
        const float wk = bb[kk * U + u];
        const float zi = ugaussian_el((float)xs[i * U + u] / divisor);
        const float tmp = s_dat[2 * D + i] * wk + s_dat[i] * zi;
        bb[l * U + u] = j == -1 ? tmp : tmp + s_dat[D + i] * bb[j * U + u];
      }
      for (int ii = 1; ii < D; ii++) {
        const int i = D - ii;
        bb[i * U + u] = bb[i * U + u] - bb[(i - 1) * U + u];
      }
    }
    // per model: correlation (:188-199), prices (:201-228), payoff (:242-301)
#pragma unroll
    for (int mm = 0; mm < kOpModels; mm++) {
      if (mm >= nm) break;
      const int m = m0 + mm;
      const float* cm = a.md_cs + (int64_t)m * U * U;
      const float* vol = a.md_vols + (int64_t)m * K;
      const float* dr = a.md_drifts + (int64_t)m * K;
      const float* st = a.md_sts + (int64_t)m * U;
      const float* disc = a.md_discts + (int64_t)m * a.num_discts;
      float sc[U];
#pragma unroll
      for (int u = 0; u < U; u++) sc[u] = 1.0f;
      float pay = 0.0f, amount = 0.0f;
      int date = 0;
      bool decided = false, cond = false;
      for (int d = 0; d < D; d++) {
        float price[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
          float noise = 0.0f;
#pragma unroll
          for (int i = 0; i <= u; i++) noise = noise + bb[d * U + i] * cm[u * U + i];
          const float cv = dr[d * U + u] + noise * vol[d * U + u];
          sc[u] = sc[u] * f32exp(cv);
          price[u] = st[u] * sc[u];
        }
        if constexpr (C == 1) {
          const float amt = (price[0] - 4000.0f) * a.md_detvals[m];
          pay = (0.0f < amt ? amt : 0.0f) * disc[0];
        } else if constexpr (C == 2) {
          if (!decided) {
            if (d < 4) {
              if (1.0f <= fmin_payoff(price)) {
                date = d;
                amount = d == 0 ? 1150.0f : d == 1 ? 1300.0f : d == 2 ? 1450.0f : 1600.0f;
                decided = true;
              }
            } else {
              const float x50 = fmin_payoff(price);
              date = 4;
              amount = 1.0f <= x50 ? 1750.0f : (0.75f < x50 ? 1000.0f : x50 * 1000.0f);
              decided = true;
            }
          }
          if (d == D - 1) pay = amount * disc[date];
        } else {
          cond = cond || (price[0] <= 2630.6349999999998f || price[1] <= 8288.0f || price[2] <= 840.0f);
          if (d == D - 1) {
            const float price1 = 100.0f * disc[0];
            const bool goto40 = cond && (price[0] < 3758.05f || price[1] < 11840.0f || price[2] < 1200.0f);
            const float amt = goto40 ? 1000.0f * fmin_payoff(price) : 1000.0f;
            pay = price1 + amt * disc[1];
          }
        }
      }
      acc[mm] += (double)pay;
      if (a.pay_out) a.pay_out[it * a.num_models + m0 + mm] = pay;
    }
  }
  // per-CTA sums in a fixed tree order: partial[mm][blockIdx.x]
  __shared__ double red[kOpThreads];
#pragma unroll
  for (int mm = 0; mm < kOpModels; mm++) {
    if (mm >= nm) break;
    red[threadIdx.x] = ok ? acc[mm] : __longlong_as_double(0x7ff8000000000000LL);
    __syncthreads();
    for (int w = kOpThreads / 2; w > 0; w >>= 1) {
      if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
      __syncthreads();
    }
    if (threadIdx.x == 0) partial[(int64_t)mm * gridDim.x + blockIdx.x] = red[0];
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Warp per path (contract 3: 367 dates x 3 underlyings)
// ---------------------------------------------------------------------------
// A warp prices a contiguous range of paths, its lanes sharing each path's
// dimensions k = lane, lane + 32, ...: the Sobol integers (kept from path to
// path), the Gaussians, the differences, the exponentials and the payoff's
// date test run across the lanes on [date][underlying] arrays in shared
// memory.  The bridge recursion (:150-165) runs level by level on the CTA's
// schedule (op_bridge_schedule): the steps of one level touch disjoint
// positions and read only values of earlier levels, so each step computes
// exactly what it computes in the sequential loop.  The running product of
// the prices (the scan of :217) stays sequential per underlying, in the
// reference's order.
constexpr int kWarpPathWarps = 7;

// Thread 0 of a CTA: level[i] of every bridge step i = 1 .. D-1 -- one more
// than the levels of the last writes of the positions it reads or writes and
// of the reads of the position it writes -- and the steps sorted by level:
// order[start[v] .. start[v + 1]) are the steps of level v, v = 1 .. nlev.
// lw, lr, level: [D] scratch; start: [D + 2].  False if an index leaves the
// path.
template <int D>
__device__ bool op_bridge_schedule(const int32_t* ind, int* lw, int* lr, int* level, int* order, int* start,
                                   int& nlev) {
  if (!bridge_indices_valid<D>(ind)) return false;
  for (int p = 0; p < D; p++) lw[p] = lr[p] = -1;
  lw[ind[0] - 1] = 0;  // step 0 writes bi[0]
  int maxl = 0;
  for (int i = 1; i < D; i++) {
    const int j = ind[D + i] - 1, k = ind[2 * D + i] - 1, l = ind[i] - 1;
    int lev = max(max(lw[k], lw[l]), lr[l]) + 1;
    if (j >= 0) lev = max(lev, lw[j] + 1);
    lev = max(lev, 1);
    level[i] = lev;
    lw[l] = lev;
    lr[k] = max(lr[k], lev);
    if (j >= 0) lr[j] = max(lr[j], lev);
    maxl = max(maxl, lev);
  }
  for (int v = 0; v <= maxl + 1; v++) start[v] = 0;
  for (int i = 1; i < D; i++) start[level[i] + 1]++;
  for (int v = 1; v <= maxl + 1; v++) start[v] += start[v - 1];
  for (int v = 0; v <= maxl; v++) lw[v] = start[v];  // insertion cursors
  for (int i = 1; i < D; i++) order[lw[level[i]]++] = i;
  nlev = maxl;
  return true;
}

template <int C>
struct OpWarpSmem {
  static constexpr int D = OpShape<C>::D, KP = (OpShape<C>::D * OpShape<C>::U + 31) / 32 * 32;
  static constexpr int kFixed = (8 * D + 2 + 3) & ~3;  // bb_inds, bb_data, order, start
  static constexpr int kWarp = 3 * KP;                 // Sobol integers, two path arrays
  static constexpr int kWords = kFixed + kWarpPathWarps * kWarp;
  static_assert(3 * D <= kWarp, "the schedule's scratch fits a warp's arrays");
};

// dirT[i][k] = dir_vs[k][i]: the direction numbers of bit i of every
// dimension, contiguous for the warp's lanes.
__global__ void op_transpose_dirs_kernel(const int32_t* __restrict__ dir_vs, int K, int B,
                                         int32_t* __restrict__ dirT) {
  const int64_t n = (int64_t)K * B;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = q / K, k = q - i * K;
    dirT[q] = dir_vs[k * B + i];
  }
}

template <int C>
__global__ void __launch_bounds__(kWarpPathWarps * 32, 2) op_paths_warp_kernel(OpDev a, const int32_t* __restrict__ dirT,
                                                                            int m0, double* __restrict__ partial) {
  using L = OpWarpSmem<C>;
  constexpr int D = OpShape<C>::D, U = OpShape<C>::U, K = D * U, KP = L::KP;
  constexpr unsigned kAll = 0xffffffffu;
  extern __shared__ float op_dyn[];
  int32_t* s_ind = reinterpret_cast<int32_t*>(op_dyn);  // bb_inds: bi, li, ri
  float* s_dat = op_dyn + 3 * D;                         // bb_data: sd, lw, rw
  int* s_order = reinterpret_cast<int*>(op_dyn + 6 * D);
  int* s_start = s_order + D;  // D + 2
  __shared__ int s_ok, s_nlev;
  __shared__ double red[kWarpPathWarps];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  float* wbase = op_dyn + L::kFixed + warp * L::kWarp;
  int32_t* sX = reinterpret_cast<int32_t*>(wbase);  // Sobol integers [K]
  float* sG = wbase + KP;                           // Gaussians, then the bridge's differences
  float* sB = wbase + 2 * KP;                       // the bridge, then exponentials and prices
  for (int i = threadIdx.x; i < 3 * D; i += blockDim.x) {
    s_ind[i] = a.bb_inds[i];
    s_dat[i] = a.bb_data[i];
  }
  __syncthreads();
  if (threadIdx.x == 0) {  // scratch: warp 0's arrays, not in use yet
    int* scr = reinterpret_cast<int*>(op_dyn + L::kFixed);
    int nl = 0;
    s_ok = op_bridge_schedule<D>(s_ind, scr, scr + D, scr + 2 * D, s_order, s_start, nl);
    s_nlev = nl;
  }
  __syncthreads();
  const bool ok = s_ok;
  const int nlev = s_nlev;
  const int64_t W = (int64_t)gridDim.x * kWarpPathWarps;
  const int64_t w = (int64_t)blockIdx.x * kWarpPathWarps + warp;
  const int64_t N = ok ? a.num_mc_it : 0;
  const int64_t lo = N * w / W, hi = N * (w + 1) / W;
  const int B = a.num_bits;
  const uint32_t bits = B >= 32 ? 0xffffffffu : ((1u << B) - 1u);
  const float divisor = ldexpf(1.0f, B);
  const int nm = min(kOpModels, a.num_models - m0);
  double acc[kOpModels];
#pragma unroll
  for (int mm = 0; mm < kOpModels; mm++) acc[mm] = 0.0;
  for (int64_t it = lo; it < hi; it++) {
    const int32_t n = (int32_t)(it + 1);
    const uint32_t gray = (uint32_t)((n >> 1) ^ n) & bits;
    const int c = __ffs(n) - 1;  // the Gray-code bit path n flips
    if (it == lo) {  // Sobol point (:13-33) from the Gray code's set bits
      for (int k = lane; k < K; k += 32) sX[k] = 0;
      for (uint32_t g = gray; g != 0u; g &= g - 1u) {
        const int32_t* row = dirT + (int64_t)(__ffs((int)g) - 1) * K;
        for (int k = lane; k < K; k += 32) sX[k] ^= row[k];
      }
    } else if (c < B) {  // or from the previous path's point
      const int32_t* row = dirT + (int64_t)c * K;
#pragma unroll 4
      for (int k = lane; k < K; k += 32) sX[k] ^= row[k];
    }
    // Gaussians (:120-136) in two passes, so neither branch runs on a
    // partly idle warp: the central branch for every dimension, queueing
    // (in sB, free until the bridge) the dimensions that need the tail
    // branch; then the queue, densely
    int32_t* queue = reinterpret_cast<int32_t*>(sB);
    int nq = 0;
    for (int k0 = 0; k0 < K; k0 += 32) {
      const int k = k0 + lane;
      bool tail = false;
      if (k < K) {
        const float dp = (float)sX[k] / divisor - 0.5f;
        if (gauss_is_central(dp)) sG[k] = gauss_central(dp);
        else tail = true;
      }
      const unsigned ball = __ballot_sync(kAll, tail);
      if (tail) queue[nq + __popc(ball & ((1u << lane) - 1u))] = k;
      nq += __popc(ball);
    }
    __syncwarp();
    for (int q = lane; q < nq; q += 32) {
      const int k = queue[q];
      sG[k] = gauss_tail((float)sX[k] / divisor - 0.5f);
    }
    __syncwarp();
    for (int k = lane; k < K; k += 32) sB[k] = 0.0f;
    __syncwarp();
    if (lane < U) sB[(s_ind[0] - 1) * U + lane] = s_dat[0] * sG[lane];
    __syncwarp();
    for (int v = 1; v <= nlev; v++) {  // the bridge (:150-165), a level at a time
      // no step of a level reads a position another step of it writes, so a
      // batch of steps loads everything before it stores
      const int s0 = s_start[v], cnt = (s_start[v + 1] - s0) * U;
      constexpr int kBatch = 4;
      for (int p0 = lane; p0 < cnt; p0 += 32 * kBatch) {
        float val[kBatch];
        int dst[kBatch];
#pragma unroll
        for (int q = 0; q < kBatch; q++) {
          const int p = p0 + 32 * q;
          dst[q] = -1;
          if (p < cnt) {
            const int i = s_order[s0 + p / U], u = p % U;
            const int j = s_ind[D + i] - 1, kk = s_ind[2 * D + i] - 1;
            const float tmp = s_dat[2 * D + i] * sB[kk * U + u] + s_dat[i] * sG[i * U + u];
            val[q] = j == -1 ? tmp : tmp + s_dat[D + i] * sB[j * U + u];
            dst[q] = (s_ind[i] - 1) * U + u;
          }
        }
#pragma unroll
        for (int q = 0; q < kBatch; q++)
          if (dst[q] >= 0) sB[dst[q]] = val[q];
      }
      __syncwarp();
    }
    for (int k = lane; k < K; k += 32)  // differences of consecutive dates (:167-175)
      sG[k] = k >= U ? sB[k] - sB[k - U] : sB[k];
    __syncwarp();
#pragma unroll
    for (int mm = 0; mm < kOpModels; mm++) {
      if (mm >= nm) break;
      const int m = m0 + mm;
      const float* cm = a.md_cs + (int64_t)m * U * U;
      const float* vol = a.md_vols + (int64_t)m * K;
      const float* dr = a.md_drifts + (int64_t)m * K;
      const float* disc = a.md_discts + (int64_t)m * a.num_discts;
      for (int k = lane; k < K; k += 32) {  // exp(drift + correlated noise * vol) (:188-215)
        const int d = k / U, u = k - d * U;
        float noise = 0.0f;
        for (int i = 0; i <= u; i++) noise = noise + sG[d * U + i] * cm[u * U + i];
        sB[k] = f32exp(dr[k] + noise * vol[k]);
      }
      __syncwarp();
      if (lane < U) {  // running product and prices (:216-218)
        const float st = a.md_sts[(int64_t)m * U + lane];
        float sc = 1.0f;
        constexpr int kBlk = 8;
        for (int d0 = 0; d0 < D; d0 += kBlk) {
          float e[kBlk];
#pragma unroll
          for (int q = 0; q < kBlk; q++) e[q] = d0 + q < D ? sB[(d0 + q) * U + lane] : 1.0f;
#pragma unroll
          for (int q = 0; q < kBlk; q++) {
            if (d0 + q < D) {
              sc = sc * e[q];
              sB[(d0 + q) * U + lane] = st * sc;
            }
          }
        }
      }
      __syncwarp();
      float pay = 0.0f;
      if constexpr (C == 3) {  // :266-292
        bool hit = false;
        for (int d = lane; d < D; d += 32) {
          const float* x = sB + d * 3;
          hit = hit || (x[0] <= 2630.6349999999998f || x[1] <= 8288.0f || x[2] <= 840.0f);
        }
        const bool cond = __any_sync(kAll, hit);
        if (lane == 0) {
          const float* last = sB + (D - 1) * 3;
          const float price1 = 100.0f * disc[0];
          const bool goto40 = cond && (last[0] < 3758.05f || last[1] < 11840.0f || last[2] < 1200.0f);
          const float amt = goto40 ? 1000.0f * fmin_payoff(last) : 1000.0f;
          pay = price1 + amt * disc[1];
        }
      }
      if (lane == 0) {
        acc[mm] += (double)pay;
        if (a.pay_out) a.pay_out[it * a.num_models + m0 + mm] = pay;
      }
      __syncwarp();  // sB is rewritten by the next model or path
    }
  }
#pragma unroll
  for (int mm = 0; mm < kOpModels; mm++) {  // the CTA's sum, warps in order
    if (mm >= nm) break;
    if (lane == 0) red[warp] = ok ? acc[mm] : __longlong_as_double(0x7ff8000000000000LL);
    __syncthreads();
    if (threadIdx.x == 0) {
      double sum = 0.0;
      for (int q = 0; q < kWarpPathWarps; q++) sum += red[q];
      partial[(int64_t)mm * gridDim.x + blockIdx.x] = sum;
    }
    __syncthreads();
  }
}

// out[m0 + mm] = (f32)(sum of partial[mm][0 .. T)) / (f32)num_mc_it, one CTA
// per model, the same order on every run (T: the paths kernel's CTAs).
constexpr int kOpReduceThreads = 256;
__global__ void __launch_bounds__(kOpReduceThreads) op_reduce_kernel(const double* __restrict__ partial, int64_t T,
                                                                     int m0, int num_mc_it, float* __restrict__ out) {
  __shared__ double red[kOpReduceThreads];
  const int mm = blockIdx.x;
  double s = 0.0;
  for (int64_t i = threadIdx.x; i < T; i += kOpReduceThreads) s += partial[(int64_t)mm * T + i];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = kOpReduceThreads / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[m0 + mm] = (float)red[0] / (float)num_mc_it;
}

// ---------------------------------------------------------------------------
// The reference's own order of the sum over paths (finpar/OptionPricing.fut:321
// as its golden outputs were produced): an f32 running sum in path order,
// s_k = fl(s_{k-1} + p_k).  Computed exactly, in parallel, from one fact: while
// s stays in one binade [2^e, 2^(e+1)) -- f32 grid spacing u = 2^(e-23) -- and
// p_k >= 0, fl(s + p_k) = s + u * t_k, where t_k is p_k / u rounded to the
// nearest integer and does not depend on s (except on an exact tie, whose
// round-to-even goes by the parity of s / u).  So a chunk of payoffs adds the
// integer sum of its t_k to s / u until the sum would leave the binade; the
// payoffs where that happens, ties, zero or tiny running sums and anything not
// a finite nonnegative normal number are added one at a time in f32, exactly
// as the sequential loop does.
// ---------------------------------------------------------------------------
constexpr int kSeqThreads = 1024;
constexpr int kSeqPer = 16;  // payoffs per thread per chunk

// t = p / 2^(e-23) rounded to nearest; false when p needs a step of its own
// (a tie, p >= 2^e, p negative, non-finite or subnormal)
__device__ __forceinline__ bool seq_units(float p, int e, uint32_t& t) {
  const uint32_t b = __float_as_uint(p);
  if (b == 0u) {  // +0
    t = 0;
    return true;
  }
  const int be = (int)((b >> 23) & 0xffu);
  if ((b >> 31) || be == 0 || be == 0xff) return false;
  const int d = e - (be - 127);  // p in [2^(e-d), 2^(e-d+1))
  if (d < 1) return false;
  const uint32_t m = (b & 0x7fffffu) | 0x800000u;
  if (d > 31) {
    t = 0;
    return true;
  }
  t = m >> d;
  const uint32_t rem = m & ((1u << d) - 1u), half = 1u << (d - 1);
  if (rem == half) return false;
  t += rem > half;
  return true;
}

__device__ __forceinline__ int64_t warp_excl_scan(int64_t v, int lane) {
  int64_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int64_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  return x - v;
}

__global__ void __launch_bounds__(kSeqThreads) op_seq_reduce_kernel(const float* __restrict__ pay, int64_t N,
                                                                    int num_models, int m0, int num_mc_it,
                                                                    float* __restrict__ out) {
  const int mm = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const float* p = pay + m0 + mm;  // path k at p[k * num_models]
  __shared__ float s_sum;
  __shared__ long long s_next;
  __shared__ int s_stop;
  __shared__ long long s_warp[kSeqThreads / 32];
  __shared__ long long s_base;
  if (tid == 0) {
    s_sum = 0.0f;
    s_next = 0;
  }
  __syncthreads();
  constexpr int CH = kSeqThreads * kSeqPer;
  while (true) {
    const int64_t i0 = s_next;
    const float s = s_sum;
    if (i0 >= N) break;
    const uint32_t sb = __float_as_uint(s);
    const int se = (int)((sb >> 23) & 0xffu);
    if (se == 0 || se == 0xff || (sb >> 31)) {  // zero, tiny or irregular running sum: one step
      __syncthreads();
      if (tid == 0) {
        s_sum = s + p[i0 * num_models];
        s_next = i0 + 1;
      }
      __syncthreads();
      continue;
    }
    const int e = se - 127;
    const int64_t S0 = (int64_t)((sb & 0x7fffffu) | 0x800000u);  // s / u
    const int64_t len = min((int64_t)CH, N - i0);
    // pass 1: the first payoff of the chunk that needs a step of its own
    if (tid == 0) s_stop = (int)len;
    __syncthreads();
    uint32_t t[kSeqPer];
    int my_stop = (int)len;
#pragma unroll
    for (int j = 0; j < kSeqPer; j++) {
      const int k = tid * kSeqPer + j;
      t[j] = 0;
      if (k < len && my_stop == (int)len && !seq_units(p[(i0 + k) * num_models], e, t[j])) my_stop = k;
    }
    if (my_stop < (int)len) atomicMin(&s_stop, my_stop);
    __syncthreads();
    const int stop = s_stop;
    // pass 2: units before the stop, scanned; the first payoff that would
    // carry the sum out of the binade is a stop too
    int64_t mine = 0;
#pragma unroll
    for (int j = 0; j < kSeqPer; j++)
      if (tid * kSeqPer + j < stop) mine += t[j];
    const int64_t wex = warp_excl_scan(mine, lane);
    if (lane == 31) s_warp[warp] = wex + mine;
    __syncthreads();
    if (warp == 0) {
      const int64_t v = lane < kSeqThreads / 32 ? s_warp[lane] : 0;
      const int64_t x = warp_excl_scan(v, lane);
      if (lane < kSeqThreads / 32) s_warp[lane] = x;
    }
    __syncthreads();
    int64_t run = S0 + s_warp[warp] + wex;  // s / u before this thread's first payoff
    const int64_t lim = (int64_t)1 << 24;   // s / u reaching 2^24 leaves the binade
    int cross = stop;
#pragma unroll
    for (int j = 0; j < kSeqPer; j++) {
      const int k = tid * kSeqPer + j;
      if (k < stop && cross == stop) {
        if (run + t[j] >= lim) cross = k; else run += t[j];
      }
    }
    if (cross < stop) atomicMin(&s_stop, cross);
    __syncthreads();
    const int q = s_stop;
    // the sum before payoff q, from the thread whose range holds q (or the last)
    const int owner = q < (int)len ? q / kSeqPer : kSeqThreads - 1;
    if (tid == owner) {
      int64_t r = S0 + s_warp[warp] + wex;
#pragma unroll
      for (int j = 0; j < kSeqPer; j++)
        if (tid * kSeqPer + j < q) r += t[j];
      s_base = r;
    }
    __syncthreads();
    if (tid == 0) {
      float v = ldexpf((float)s_base, e - 23);  // exact: s_base < 2^24
      int64_t nx = i0 + len;
      if (q < (int)len) {
        v = v + p[(i0 + q) * num_models];  // the step the sequential loop takes there
        nx = i0 + q + 1;
      }
      s_sum = v;
      s_next = nx;
    }
    __syncthreads();
  }
  if (tid == 0) {
    const float f64_order = out[m0 + mm];  // NaN when the paths kernel priced nothing (bad bridge)
    out[m0 + mm] = f64_order != f64_order ? f64_order : s_sum / (float)num_mc_it;
  }
}

constexpr size_t kWarpSmem3 = sizeof(float) * OpWarpSmem<3>::kWords;

// CTAs of the paths kernel for `paths` paths of contract c: eight 128-thread
// CTAs per SM (thread per path), or two 7-warp CTAs per SM (warp per path,
// contract 3); fewer when there are fewer paths.
int64_t op_ctas(const futhark_context* ctx, int c, int64_t paths) {
  const int64_t per = c == 3 ? kWarpPathWarps : kOpThreads;  // paths a CTA takes at once
  const int64_t want = (int64_t)ctx->num_sms * (c == 3 ? 2 : 8);
  return std::max<int64_t>(1, std::min(want, (paths + per - 1) / per));
}
constexpr int kOpMaxCtasPerSm = 8;

// Shapes and sizes of one pricing (lock held); the message names the failure.
int op_validate(futhark_context* ctx, const op_args* q) {
  const int c = q->contract_number;
  if (q->num_models < 0 || q->num_und < 0 || q->num_dates < 0 || q->num_discts < 0 || q->num_bits < 0)
    return set_error(ctx, FUTHARK_PROGRAM_ERROR, "option pricing: negative dimension");
  if (q->num_mc_it < 0)  // iota of a negative length (:315)
    return set_error(ctx, FUTHARK_PROGRAM_ERROR, "option pricing: negative num_mc_it");
  if (q->num_bits > 32)
    return set_error(ctx, FUTHARK_PROGRAM_ERROR, "option pricing: num_bits above 32 is not supported");
  const int need_d[4] = {0, 1, 5, 367}, need_u[4] = {0, 1, 3, 3}, need_disc[4] = {0, 1, 5, 2};
  if (c >= 1 && c <= 3 && q->num_models > 0) {
    if (q->num_dates != need_d[c] || q->num_und != need_u[c])
      return set_error(ctx, FUTHARK_PROGRAM_ERROR,
                       "option pricing: contract " + std::to_string(c) + " needs [" + std::to_string(need_d[c]) +
                           "][" + std::to_string(need_u[c]) + "] paths (size coercion failed)");
    if (q->num_discts < need_disc[c])
      return set_error(ctx, FUTHARK_PROGRAM_ERROR, "option pricing: too few discount factors for the contract");
  }
  return 0;
}

// Scratch: the CTAs' partial sums, then (contract 3) the transposed
// direction numbers.
size_t partial_bytes(const futhark_context* ctx) {
  return (sizeof(double) * (size_t)kOpModels * (size_t)ctx->num_sms * kOpMaxCtasPerSm + 255) & ~(size_t)255;
}
size_t dirs_bytes(const op_args* q) {
  const size_t dirs = q->contract_number == 3
                          ? sizeof(int32_t) * (size_t)std::max(0, q->num_dates) * std::max(0, q->num_und) *
                                std::max(0, q->num_bits)
                          : 0;
  return (dirs + 255) & ~(size_t)255;
}
// (reference order) every path's payoff, [path][model]
size_t payoff_bytes(const futhark_context* ctx, const op_args* q) {
  if (ctx->reduce_order != 1) return 0;
  return sizeof(float) * (size_t)std::max(0, q->num_mc_it) * (size_t)std::max(0, q->num_models);
}
size_t scratch_for(const futhark_context* ctx, const op_args* q) {
  return partial_bytes(ctx) + dirs_bytes(q) + payoff_bytes(ctx, q) + 256;
}

// Enqueues one pricing (lock held, device set, shapes valid, scratch large enough).
int op_launch(futhark_context* ctx, const op_args* q, float* out, void* scratch) {
  if (q->num_models == 0) return 0;
  const int c = q->contract_number;
  const bool priced = c >= 1 && c <= 3 && q->num_mc_it > 0;
  float* pay_out = priced && ctx->reduce_order == 1
                       ? reinterpret_cast<float*>(static_cast<char*>(scratch) + partial_bytes(ctx) + dirs_bytes(q))
                       : nullptr;
  OpDev a{q->num_mc_it, q->num_bits, q->num_models, q->num_discts, q->dir_vs, q->md_cs, q->md_vols, q->md_drifts,
          q->md_sts, q->md_detvals, q->md_discts, q->bb_inds, q->bb_data, pay_out};
  double* partial = static_cast<double*>(scratch);
  const int64_t T = priced ? op_ctas(ctx, c, q->num_mc_it) : 0;  // CTAs, one partial each
  int32_t* dirT = reinterpret_cast<int32_t*>(static_cast<char*>(scratch) + partial_bytes(ctx));
  if (priced && c == 3) {
    cudaError_t e = cudaFuncSetAttribute((const void*)op_paths_warp_kernel<3>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kWarpSmem3);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "option pricing attributes");
    const int64_t kb = (int64_t)q->num_dates * q->num_und * q->num_bits;
    op_transpose_dirs_kernel<<<(unsigned)std::max<int64_t>(1, std::min<int64_t>((kb + 255) / 256, 1024)), 256, 0,
                               ctx->stream>>>(q->dir_vs, q->num_dates * q->num_und, q->num_bits, dirT);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(ctx, e, "option pricing transpose launch");
  }
  for (int m0 = 0; m0 < q->num_models; m0 += kOpModels) {
    const int nm = std::min(kOpModels, q->num_models - m0);
    if (priced) {
      if (c == 1) op_paths_kernel<1><<<(unsigned)T, kOpThreads, 0, ctx->stream>>>(a, m0, partial);
      else if (c == 2) op_paths_kernel<2><<<(unsigned)T, kOpThreads, 0, ctx->stream>>>(a, m0, partial);
      else
        op_paths_warp_kernel<3><<<(unsigned)T, kWarpPathWarps * 32, kWarpSmem3, ctx->stream>>>(a, dirT, m0, partial);
      const cudaError_t e = cudaGetLastError();
      if (e != cudaSuccess) return cuda_fail(ctx, e, "option pricing launch");
    }
    // other contracts price every path at 0 (:302); no paths gives 0 / 0
    op_reduce_kernel<<<nm, kOpReduceThreads, 0, ctx->stream>>>(partial, T, m0, q->num_mc_it, out);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(ctx, e, "option pricing reduction launch");
    if (pay_out) {  // the reference's order replaces the f64 one (NaN stays NaN)
      op_seq_reduce_kernel<<<nm, kSeqThreads, 0, ctx->stream>>>(pay_out, q->num_mc_it, q->num_models, m0,
                                                                 q->num_mc_it, out);
      e = cudaGetLastError();
      if (e != cudaSuccess) return cuda_fail(ctx, e, "option pricing ordered reduction launch");
    }
  }
  return 0;
}

}  // namespace

extern "C" {

FUT_ARRAY_API(f32_1d, float, 1, int64_t dim0)
FUT_ARRAY_API(f32_2d, float, 2, int64_t dim0, int64_t dim1)
FUT_ARRAY_API(f32_3d, float, 3, int64_t dim0, int64_t dim1, int64_t dim2)
FUT_ARRAY_API(i32_2d, int32_t, 2, int64_t dim0, int64_t dim1)

int futhark_entry_main(struct futhark_context* ctx, struct futhark_f32_1d** out0, int32_t contract_number,
                       int32_t num_mc_it, const struct futhark_i32_2d* dir_vs, const struct futhark_f32_3d* md_cs,
                       const struct futhark_f32_3d* md_vols, const struct futhark_f32_3d* md_drifts,
                       const struct futhark_f32_2d* md_sts, const struct futhark_f32_2d* md_detvals,
                       const struct futhark_f32_2d* md_discts, const struct futhark_i32_2d* bb_inds,
                       const struct futhark_f32_2d* bb_data) {
  std::lock_guard<std::mutex> g(ctx->mu);
  if (!ctx->ok) return set_error(ctx, FUTHARK_PROGRAM_ERROR, "context has no usable CUDA device");
  if (!out0 || !dir_vs || !md_cs || !md_vols || !md_drifts || !md_sts || !md_detvals || !md_discts || !bb_inds ||
      !bb_data)
    return set_error(ctx, FUTHARK_PROGRAM_ERROR, "null array");
  const int64_t M = md_vols->shape[0], D = md_vols->shape[1], U = md_vols->shape[2];
  const int64_t B = dir_vs->shape[1], ND = md_discts->shape[1];
  // the entry point's size parameters (OptionPricing.fut:304-314)
  const bool sizes_ok = dir_vs->shape[0] == D * U && md_cs->shape[0] == M && md_cs->shape[1] == U &&
                        md_cs->shape[2] == U && md_drifts->shape[0] == M && md_drifts->shape[1] == D &&
                        md_drifts->shape[2] == U && md_sts->shape[0] == M && md_sts->shape[1] == U &&
                        md_detvals->shape[0] == M && md_detvals->shape[1] == 1 && md_discts->shape[0] == M &&
                        bb_inds->shape[0] == 3 && bb_inds->shape[1] == D && bb_data->shape[0] == 3 &&
                        bb_data->shape[1] == D;
  if (!sizes_ok) return set_error(ctx, FUTHARK_PROGRAM_ERROR, "option pricing: input sizes do not match");
  if (M > INT32_MAX || D > INT32_MAX || U > INT32_MAX || B > INT32_MAX || ND > INT32_MAX)
    return set_error(ctx, FUTHARK_PROGRAM_ERROR, "option pricing: dimension too large");
  op_args q{contract_number, num_mc_it, (int32_t)B, (int32_t)M, (int32_t)U, (int32_t)D, (int32_t)ND,
            dir_vs->data, md_cs->data, md_vols->data, md_drifts->data, md_sts->data, md_detvals->data,
            md_discts->data, bb_inds->data, bb_data->data};
  int rc = op_validate(ctx, &q);
  if (rc) return rc;
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "option pricing");
  // the bridge's indices select dates (:155-169, unchecked in the reference)
  if (contract_number >= 1 && contract_number <= 3 && M > 0 && D > 0) {
    std::vector<int32_t> ind(3 * D);
    e = cudaMemcpyAsync(ind.data(), bb_inds->data, sizeof(int32_t) * ind.size(), cudaMemcpyDeviceToHost,
                        ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "option pricing: reading bb_inds");
    // bi[i] for every i; li[i] (0: no left point) and ri[i] from i = 1 on
    bool in_range = ind[0] >= 1 && ind[0] <= D;
    for (int64_t i = 1; i < D; i++)
      in_range = in_range && ind[i] >= 1 && ind[i] <= D && ind[D + i] >= 0 && ind[D + i] <= D &&
                 ind[2 * D + i] >= 1 && ind[2 * D + i] <= D;
    if (!in_range)
      return set_error(ctx, FUTHARK_PROGRAM_ERROR, "option pricing: bb_inds selects a date outside the path");
  }
  const int64_t d1[1] = {M};
  futhark_f32_1d* out = alloc_array<futhark_f32_1d>(d1, 1);
  if (!out || !ensure_scratch(ctx, scratch_for(ctx, &q))) {
    drop_array(out);
    return set_error(ctx, FUTHARK_OUT_OF_MEMORY, "out of device memory");
  }
  rc = op_launch(ctx, &q, out->data, ctx->scratch);
  if (!rc) {
    e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) rc = cuda_fail(ctx, e, "option pricing");
  }
  if (rc) {
    drop_array(out);
    return rc;
  }
  *out0 = out;
  return 0;
}

size_t op_scratch_bytes(struct futhark_context* ctx, const struct op_args* args) {
  if (!ctx || !args || !ctx->ok) return 0;
  return scratch_for(ctx, args);
}
int op_price_f32(struct futhark_context* ctx, const struct op_args* args, float* out, void* scratch) {
  std::lock_guard<std::mutex> g(ctx->mu);
  if (!ctx->ok) return set_error(ctx, FUTHARK_PROGRAM_ERROR, "context has no usable CUDA device");
  if (!args || (!out && args->num_models > 0)) return set_error(ctx, FUTHARK_PROGRAM_ERROR, "null argument");
  int rc = op_validate(ctx, args);
  if (rc) return rc;
  if (((uintptr_t)scratch & 255) != 0)
    return set_error(ctx, FUTHARK_PROGRAM_ERROR, "option pricing: scratch is not on a 256-byte boundary");
  const cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "option pricing");
  return op_launch(ctx, args, out, scratch);
}
int op_check(struct futhark_context* ctx) {
  std::lock_guard<std::mutex> g(ctx->mu);
  if (!ctx->ok) return set_error(ctx, FUTHARK_PROGRAM_ERROR, "context has no usable CUDA device");
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e == cudaSuccess) e = cudaGetLastError();
  return e == cudaSuccess ? 0 : cuda_fail(ctx, e, "option pricing");
}
void* op_context_stream(struct futhark_context* ctx) { return ctx && ctx->ok ? (void*)ctx->stream : nullptr; }
int op_context_set_reduction_order(struct futhark_context* ctx, int32_t order) {
  if (!ctx) return FUTHARK_PROGRAM_ERROR;
  std::lock_guard<std::mutex> g(ctx->mu);
  if (order != OP_ORDER_F64 && order != OP_ORDER_SEQUENTIAL_F32)
    return set_error(ctx, FUTHARK_PROGRAM_ERROR, "option pricing: unknown reduction order");
  ctx->reduce_order = order;
  return 0;
}

}  // extern "C"
