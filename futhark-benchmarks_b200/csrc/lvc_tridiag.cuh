// Batched tridiagonal solvers: the tridagNested* entry points of
// misc/ocean-sim/tridiag-test.fut:14-26 (f32, one system per row of
// [rows][m] arrays).
//
//   FORM 0  tridagSeq (misc/ocean-sim/tridiag.fut:81-95): normalised Thomas.
//   FORM 1  tridagPar (misc/ocean-sim/tridiag.fut:4-79): the three scans --
//           4-tuple matrix scan for the pivots, two linear-function scans --
//           folded left to right.
//
// Four kernels, one thread per system in each: for m up to 256 (the
// benchmark's 115 among them) lvc_tridag_tmem_kernel streams a warp's 32
// systems through shared-memory windows and keeps the row intermediates in
// tensor memory, and lvc_tridag_tma_kernel does the same with the windows
// of the CTA's 128 systems brought in by tensor copies (odd m, rows a
// multiple of 4); for m up to 400 lvc_tridag_stream_kernel streams them the
// same way and keeps the intermediates in shared memory; lvc_tridag_kernel
// (any m) reads rows in place.  All four take both forms.
// Each recurrence runs in the reference's operation
// order with every product, sum and quotient explicitly rounded (no fused
// multiply-add), so a system's solution is bit for bit the one the CPU
// restatement of the same fold gives.  The work is a handful of operations per
// element against 20 bytes of HBM traffic (four inputs, one output): the kernel
// is bound by HBM and by the latency of the sequential recurrence, which the
// many independent systems of a batch hide.  lvc_tridag_kernel keeps its
// per-row scratch (the pivots of FORM 1, the normalised super-diagonal of
// FORM 0) in a global [element][row] buffer -- consecutive threads at
// consecutive addresses -- and the right-hand side of the backward pass in the
// output row itself.
#pragma once

#include <cuda.h>  // CUtensorMap

#include <cstdint>

#include "lvc_line.cuh"  // mbarrier and bulk-copy helpers

namespace lvc {

// Raised by a bounded wait that gave up (lvc_wait_selftest_kernel below);
// reset and read by the host after each solve and self-test.
__device__ int lvc_tridag_err;

constexpr int kTriThreads = 128;  // threads (systems) per CTA of lvc_tridag_kernel

// Self-test of the bounded wait that the rollback kernels' bulk-copy and
// cluster waits use (mbar_wait): one warp waits on a fresh mbarrier for at
// most `polls` polls.  With arrive == 0 nothing ever completes its phase (no
// copy targets it and no thread arrives), so the wait runs out and the kernel
// raises lvc_tridag_err, which the host reports as a timed-out wait; with
// arrive != 0 lane 0 arrives first and the wait succeeds.  No asynchronous
// operation is in flight either way, so the CTA may exit at once.
__global__ void lvc_wait_selftest_kernel(int polls, int arrive) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncwarp();
  if (arrive && threadIdx.x == 0)
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(&bar)) : "memory");
  const bool ok = mbar_wait(&bar, 0, polls);
  if (!ok && threadIdx.x == 0) atomicExch(&lvc_tridag_err, 1);
}

__device__ __forceinline__ float tri_mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float tri_add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float tri_sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float tri_div(float a, float b) { return __fdiv_rn(a, b); }
// 1 / x correctly rounded: the same value as tri_div(1.0f, x), cheaper
__device__ __forceinline__ float tri_rcp(float x) { return __frcp_rn(x); }
// a / b correctly rounded from rb = 1 / (double)b correctly rounded in
// double: the float nearest the double product a * rb.  The product is
// within 2^-52 of a / b relatively; a quotient of two floats is never a
// point halfway between two floats nor closer to one than 2^-49 relatively
// (a nonzero multiple of a power of two over a 24-bit divisor significand),
// so the product rounds to float as a / b does.  Zeros, infinities and signs
// follow from the IEEE operations.  One double reciprocal then serves every
// quotient by the same divisor.
__device__ __forceinline__ double tri_rcpd(float b) { return __drcp_rn((double)b); }
__device__ __forceinline__ float tri_divr(float a, double rb) { return __double2float_rn(__dmul_rn((double)a, rb)); }

template <int FORM>
__global__ void __launch_bounds__(kTriThreads) lvc_tridag_kernel(int64_t rows, int m, const float* __restrict__ a,
                                                                const float* __restrict__ b,
                                                                const float* __restrict__ c,
                                                                const float* __restrict__ y,
                                                                float* __restrict__ out,
                                                                float* __restrict__ gscratch) {
  const int64_t r = (int64_t)blockIdx.x * kTriThreads + threadIdx.x;
  if (r >= rows) return;  // no barrier below: threads are independent
  const float* ar = a + r * m;
  const float* br = b + r * m;
  const float* cr = c + r * m;
  const float* yr = y + r * m;
  float* o = out + r * m;
  float* scr = gscratch + r;
  const int64_t sstride = rows;  // element i of this row's scratch at scr[i * sstride]

  if constexpr (FORM == 0) {
    // forward: cp_i = c_i / (b_i - a_i cp_{i-1}), yp_i = (y_i - a_i yp_{i-1}) / (...)  (:82-91)
    float cp = tri_div(cr[0], br[0]);
    float yp = tri_div(yr[0], br[0]);
    scr[0] = cp;
    o[0] = yp;
    for (int i = 1; i < m; i++) {
      const float ai = ar[i];
      const float nf = tri_rcp(tri_sub(br[i], tri_mul(ai, cp)));
      cp = tri_mul(cr[i], nf);
      yp = tri_mul(tri_sub(yr[i], tri_mul(ai, yp)), nf);
      scr[i * sstride] = cp;
      o[i] = yp;
    }
    // backward: x_i = yp_i - cp_i x_{i+1}  (:92-95)
    float x = yp;
    for (int i = m - 2; i >= 0; i--) {
      x = tri_sub(o[i], tri_mul(scr[i * sstride], x));
      o[i] = x;
    }
  } else {
    // Recurrence 1 (:9-33): b'_i from the scan of (b_i, -a_i c_{i-1}, 1, 0)
    const float b0 = br[0];
    float s0 = 1.0f, s1 = 0.0f, s2 = 0.0f, s3 = 1.0f;
    for (int i = 0; i < m; i++) {
      float m0 = 1.0f, m1 = 0.0f, m2 = 0.0f, m3 = 1.0f;
      if (0 < i) {
        m0 = br[i];
        m1 = tri_sub(0.0f, tri_mul(ar[i], cr[i - 1]));
        m2 = 1.0f;
        m3 = 0.0f;
      }
      const float value = tri_rcp(tri_mul(s0, m0));
      const float n0 = tri_mul(tri_add(tri_mul(m0, s0), tri_mul(m1, s2)), value);
      const float n1 = tri_mul(tri_add(tri_mul(m0, s1), tri_mul(m1, s3)), value);
      const float n2 = tri_mul(tri_add(tri_mul(m2, s0), tri_mul(m3, s2)), value);
      const float n3 = tri_mul(tri_add(tri_mul(m2, s1), tri_mul(m3, s3)), value);
      s0 = n0;
      s1 = n1;
      s2 = n2;
      s3 = n3;
      scr[i * sstride] = tri_div(tri_add(tri_mul(s0, b0), s1), tri_add(tri_mul(s2, b0), s3));
    }
    // Recurrence 2 (:38-56): y'_i = y_i - (a_i / b'_{i-1}) y'_{i-1}, into the output row
    const float y0 = yr[0];
    float c0 = 0.0f, c1 = 1.0f;
    for (int i = 0; i < m; i++) {
      float l0 = 0.0f, l1 = 1.0f;
      if (0 < i) {
        l0 = yr[i];
        l1 = tri_sub(0.0f, tri_div(ar[i], scr[(i - 1) * sstride]));
      }
      const float n0 = tri_add(l0, tri_mul(l1, c0));
      const float n1 = tri_mul(c1, l1);
      c0 = n0;
      c1 = n1;
      o[i] = tri_add(c0, tri_mul(c1, y0));
    }
    // Recurrence 3 (:61-79): backward, over the reversed index
    const float yn = tri_div(o[m - 1], scr[(int64_t)(m - 1) * sstride]);
    c0 = 0.0f;
    c1 = 1.0f;
    for (int k = 0; k < m; k++) {
      const int i = m - k - 1;
      float l0 = 0.0f, l1 = 1.0f;
      if (0 < k) {
        const float bi = scr[i * sstride];
        l0 = tri_div(o[i], bi);
        l1 = tri_sub(0.0f, tri_div(cr[i], bi));
      }
      const float n0 = tri_add(l0, tri_mul(l1, c0));
      const float n1 = tri_mul(c1, l1);
      c0 = n0;
      c1 = n1;
      o[i] = tri_add(c0, tri_mul(c1, yn));
    }
  }
}

constexpr int kTriMaxM = 400;  // the streaming kernel's limit: 2 x 32 x 401 floats + windows = 112 KB

// Streaming kernel (both forms of lvc_tridag_kernel; used where the tensor-
// memory kernel does not fit, 256 < m <= 400): one warp per 32 consecutive
// systems, lane = system, but the four input rows are not staged whole.
// They pass through a double-buffered window of kTriWin columns (cp.async,
// 4-byte copies: 8 lanes cover 8 consecutive columns of one row, so a
// warp's copy instruction reads 4 short runs), and shared memory keeps only
// the two intermediates the backward pass needs per row -- FORM 0: cp_i and
// yp_i; FORM 1: b'_i and y'_i (c_i comes through the window a second time,
// last column first) -- half of what staging the four input rows would take,
// so twice the systems are in flight.  The arithmetic and its order are those
// of lvc_tridag_kernel (FORM 1's recurrences 1 and 2 fused into one forward
// pass over i: each step reads only values the pass has already produced).
// The solution overwrites the second intermediate and leaves row by row,
// consecutive lanes on consecutive elements.
constexpr int kTriWin = 8;

__device__ __forceinline__ void cp_async4(float* dst, const float* src, bool valid) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(smem_u32(dst)), "l"(src),
               "r"(valid ? 4 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Shared floats per warp: the two row arrays (row stride m | 1: lane = row
// reads conflict-free) and 2 windows x 4 arrays x 32 rows x (kTriWin + 1).
__host__ __device__ __forceinline__ int tri_stream_ld(int m) { return m | 1; }
__host__ __device__ __forceinline__ int64_t tri_stream_floats(int m) {
  return 2LL * 32 * tri_stream_ld(m) + 2LL * 4 * 32 * (kTriWin + 1);
}

template <int FORM>
__global__ void __launch_bounds__(32) lvc_tridag_stream_kernel(int64_t rows, int m, const float* __restrict__ a,
                                                              const float* __restrict__ b,
                                                              const float* __restrict__ c,
                                                              const float* __restrict__ y,
                                                              float* __restrict__ out) {
  extern __shared__ __align__(16) float tri_s[];
  const int lane = threadIdx.x;
  const int64_t r0 = (int64_t)blockIdx.x * 32;
  const int nr = (int)(rows - r0 < 32 ? rows - r0 : 32);
  const int ld = tri_stream_ld(m);
  float* P = tri_s;            // cp_i (FORM 0) or b'_i (FORM 1), [32][ld]
  float* Q = P + 32 * ld;      // yp_i or y'_i, then x_i
  float* Wn = Q + 32 * ld;     // [2][4][32][kTriWin + 1]
  constexpr int WS = kTriWin + 1, WA = 32 * WS, WB = 4 * WA;
  const float* src[4] = {a, b, c, y};
  const int nq = (m + kTriWin - 1) / kTriWin;
  // chunk q of the arrays in `mask` into window buffer `buf`: 8 lanes per row
  // segment, 4 rows per copy instruction
  auto fetch = [&](int q, int buf, int mask) {
#pragma unroll
    for (int arr = 0; arr < 4; arr++) {
      if (!((mask >> arr) & 1)) continue;
#pragma unroll
      for (int t = 0; t < 32 * kTriWin / 32; t++) {
        const int idx = t * 32 + lane, row = idx / kTriWin, col = idx % kTriWin;
        const int gcol = q * kTriWin + col;
        const bool valid = row < nr && gcol < m;
        const float* g = valid ? src[arr] + (r0 + row) * (int64_t)m + gcol : src[arr];
        cp_async4(Wn + buf * WB + arr * WA + row * WS + col, g, valid);
      }
    }
    cp_async_commit();
  };
  if constexpr (FORM == 0) {
    // forward: cp_i = c_i / (b_i - a_i cp_{i-1}), yp_i = (y_i - a_i yp_{i-1}) / (...)  (:82-91)
    float cp = 0.0f, yp = 0.0f;
    fetch(0, 0, 15);
    for (int q = 0; q < nq; q++) {
      if (q + 1 < nq) {
        fetch(q + 1, (q + 1) & 1, 15);
        cp_async_wait<1>();
      } else {
        cp_async_wait<0>();
      }
      __syncwarp();
      const float* w = Wn + (q & 1) * WB + lane * WS;
      if (lane < nr) {
#pragma unroll
        for (int k = 0; k < kTriWin; k++) {
          const int i = q * kTriWin + k;
          if (i < m) {
            const float ai = w[k], bi = w[WA + k], ci = w[2 * WA + k], yi = w[3 * WA + k];
            if (i == 0) {
              cp = tri_div(ci, bi);
              yp = tri_div(yi, bi);
            } else {
              const float nf = tri_rcp(tri_sub(bi, tri_mul(ai, cp)));
              cp = tri_mul(ci, nf);
              yp = tri_mul(tri_sub(yi, tri_mul(ai, yp)), nf);
            }
            P[lane * ld + i] = cp;
            Q[lane * ld + i] = yp;
          }
        }
      }
      __syncwarp();  // the window is refilled two chunks on
    }
    // backward: x_i = yp_i - cp_i x_{i+1}  (:92-95)
    if (lane < nr) {
      float x = Q[lane * ld + m - 1];
      for (int i = m - 2; i >= 0; i--) {
        x = tri_sub(Q[lane * ld + i], tri_mul(P[lane * ld + i], x));
        Q[lane * ld + i] = x;
      }
    }
  } else {
    // Recurrences 1 and 2 in one forward pass: b'_i from the 4-tuple scan of
    // (b_i, -a_i c_{i-1}, 1, 0), then y'_i from the 2-tuple scan of
    // (y_i, -a_i / b'_{i-1}); both as lvc_tridag_kernel computes them.
    float s0 = 1.0f, s1 = 0.0f, s2 = 0.0f, s3 = 1.0f, b0 = 0.0f, cprev = 0.0f;
    float y0 = 0.0f, c0 = 0.0f, c1 = 1.0f, bprev = 0.0f;
    fetch(0, 0, 15);
    for (int q = 0; q < nq; q++) {
      if (q + 1 < nq) {
        fetch(q + 1, (q + 1) & 1, 15);
        cp_async_wait<1>();
      } else {
        cp_async_wait<0>();
      }
      __syncwarp();
      const float* w = Wn + (q & 1) * WB + lane * WS;
      if (lane < nr) {
  #pragma unroll
        for (int k = 0; k < kTriWin; k++) {
          const int i = q * kTriWin + k;
          if (i < m) {
            const float ai = w[k], bi = w[WA + k], ci = w[2 * WA + k], yi = w[3 * WA + k];
            if (i == 0) {
              b0 = bi;
              y0 = yi;
            }
            float m0 = 1.0f, m1 = 0.0f, m2 = 0.0f, m3 = 1.0f;
            if (0 < i) {
              m0 = bi;
              m1 = tri_sub(0.0f, tri_mul(ai, cprev));
              m2 = 1.0f;
              m3 = 0.0f;
            }
            cprev = ci;
            const float value = tri_rcp(tri_mul(s0, m0));
            const float n0 = tri_mul(tri_add(tri_mul(m0, s0), tri_mul(m1, s2)), value);
            const float n1 = tri_mul(tri_add(tri_mul(m0, s1), tri_mul(m1, s3)), value);
            const float n2 = tri_mul(tri_add(tri_mul(m2, s0), tri_mul(m3, s2)), value);
            const float n3 = tri_mul(tri_add(tri_mul(m2, s1), tri_mul(m3, s3)), value);
            s0 = n0;
            s1 = n1;
            s2 = n2;
            s3 = n3;
            const float bpi = tri_div(tri_add(tri_mul(s0, b0), s1), tri_add(tri_mul(s2, b0), s3));  // b'_i
            float l0 = 0.0f, l1 = 1.0f;
            if (0 < i) {
              l0 = yi;
              l1 = tri_sub(0.0f, tri_div(ai, bprev));
            }
            const float e0 = tri_add(l0, tri_mul(l1, c0));
            const float e1 = tri_mul(c1, l1);
            c0 = e0;
            c1 = e1;
            P[lane * ld + i] = bpi;
            Q[lane * ld + i] = tri_add(c0, tri_mul(c1, y0));  // y'_i
            bprev = bpi;
          }
        }
      }
      __syncwarp();
    }
    // Recurrence 3, backward, with c_i through the window again (last chunk first)
    float yn = 0.0f;
    if (lane < nr) yn = tri_div(Q[lane * ld + m - 1], P[lane * ld + m - 1]);
    c0 = 0.0f;
    c1 = 1.0f;
    fetch(nq - 1, 0, 4);
    for (int qq = 0; qq < nq; qq++) {
      const int q = nq - 1 - qq;
      if (qq + 1 < nq) {
        fetch(q - 1, (qq + 1) & 1, 4);
        cp_async_wait<1>();
      } else {
        cp_async_wait<0>();
      }
      __syncwarp();
      const float* w = Wn + (qq & 1) * WB + lane * WS;
      if (lane < nr) {
  #pragma unroll
        for (int kk = kTriWin - 1; kk >= 0; kk--) {
          const int i = q * kTriWin + kk;
          if (i < m) {
            float l0 = 0.0f, l1 = 1.0f;
            if (i < m - 1) {
              const float bi = P[lane * ld + i];
              l0 = tri_div(Q[lane * ld + i], bi);
              l1 = tri_sub(0.0f, tri_div(w[2 * WA + kk], bi));
            }
            const float n0 = tri_add(l0, tri_mul(l1, c0));
            const float n1 = tri_mul(c1, l1);
            c0 = n0;
            c1 = n1;
            Q[lane * ld + i] = tri_add(c0, tri_mul(c1, yn));
          }
        }
      }
      __syncwarp();
    }
  }
  __syncwarp();
  // the solution rows (Q, stride ld) to out, consecutive lanes on consecutive elements
  float* dst = out + r0 * (int64_t)m;
  const int64_t n = (int64_t)nr * m;
  if (ld == m) {
    for (int64_t e = lane; e < n; e += 32) __stcs(dst + e, Q[e]);
  } else {
    for (int64_t e = lane; e < n; e += 32) {
      const int rr = (int)(e / m), cc = (int)(e - (int64_t)rr * m);
      __stcs(dst + e, Q[rr * ld + cc]);
    }
  }
}

// ---------------------------------------------------------------------------
// Tensor-memory kernel (m <= 256): the row intermediates live in TMEM.
// ---------------------------------------------------------------------------
// The streaming kernel above is bound by the latency of each system's
// sequential chain at the few warps per SM that shared memory leaves it (two
// intermediate rows of 32 systems per warp).
// Here the intermediates go to tensor memory instead -- 256 KB per SM that
// nothing else of this library uses: thread t of a warp owns TMEM lane
// 32 (warp % 4) + t of its CTA's allocation, and the two 32-bit values of
// element i (FORM 0: cp_i, yp_i; FORM 1: the quotients y'_i / b'_i and
// -c_i / b'_i that the backward recurrence folds) sit in columns 2i, 2i + 1,
// written and read as 16-column rows by tcgen05.st / tcgen05.ld, one per
// window of eight elements.  Shared memory keeps only the input ring (three
// stages of kTriWin-column windows of the four inputs, cp.async) and an
// output window, so a 4-warp CTA needs 60 KB and, for m <= 128, 256 TMEM
// columns: two CTAs, eight warps, per SM; for m <= 256, 512 columns: one CTA
// per SM.  The shared-memory request is padded -- 80 KB for 256 columns,
// 150 KB for 512 -- so that whatever mix of these CTAs an SM holds, even
// from concurrent launches, asks for at most its 512 columns and no CTA
// waits in tcgen05.alloc.  The arithmetic and its
// order are lvc_tridag_kernel's, with FORM 1's three recurrences fused into
// the forward pass and the backward fold.
constexpr int kTriTmemWarps = 4;
constexpr int kTriTmemMaxM = 256;  // 16 columns per window of 8: 512 columns
constexpr int kTriTmemStages = 3;
// TMEM columns of a CTA for inner size m (a power of two, 256 or 512)
__host__ __device__ __forceinline__ int tri_tmem_cols(int m) { return m <= 128 ? 256 : 512; }
__host__ __device__ __forceinline__ size_t tri_tmem_smem(int cols) {
  const size_t need = 16 + sizeof(float) * kTriTmemWarps * (kTriTmemStages * 4 * 32 * (kTriWin + 1) + 32 * (kTriWin + 1));
  const size_t pad = cols > 256 ? 150 * 1024 : 80 * 1024;  // 150 + 80 KB exceed an SM's 228 KB
  return need > pad ? need : pad;
}

__device__ __forceinline__ void tmem_alloc(uint32_t* dst, int ncols) {  // whole warp
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(dst)), "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {  // whole warp
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, int ncols) {  // whole warp
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tmem_fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
}
__device__ __forceinline__ void tmem_fence_after_sync() {
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
}
// 16 consecutive 32-bit columns of this thread's lane (whole warp)
__device__ __forceinline__ void tmem_st16(uint32_t taddr, const float (&v)[16]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16};\n" ::"r"(taddr),
      "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])), "r"(__float_as_uint(v[3])),
      "r"(__float_as_uint(v[4])), "r"(__float_as_uint(v[5])), "r"(__float_as_uint(v[6])), "r"(__float_as_uint(v[7])),
      "r"(__float_as_uint(v[8])), "r"(__float_as_uint(v[9])), "r"(__float_as_uint(v[10])),
      "r"(__float_as_uint(v[11])), "r"(__float_as_uint(v[12])), "r"(__float_as_uint(v[13])),
      "r"(__float_as_uint(v[14])), "r"(__float_as_uint(v[15]))
      : "memory");
}
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;\n" ::: "memory"); }
// the load and its wait in one statement, so no use of the values can be
// scheduled before they have arrived (whole warp)
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];\n"
      "tcgen05.wait::ld.sync.aligned;\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int k = 0; k < 16; k++) v[k] = __uint_as_float(r[k]);
}

// The forward state of one system (FORM 0: cp, yp; FORM 1: the 4-tuple
// scan s, b_0, c_{i-1}, the linear scan (c0, c1), y_0, 1 / b'_{i-1}, and the
// last quotient y'_{m-1} / b'_{m-1} that starts the backward fold).
struct TriFwd {
  float cp = 0.0f, yp = 0.0f;
  float s0 = 1.0f, s1 = 0.0f, s2 = 0.0f, s3 = 1.0f, b0 = 0.0f, cprev = 0.0f;
  float y0 = 0.0f, c0 = 0.0f, c1 = 1.0f, yn = 0.0f;
  double rbprev = 0.0;  // 1 / b'_{i-1}, correctly rounded in double (tri_divr)
};

// Window q (elements q * kTriWin + k) of a system's forward pass, its inputs
// a, b, c, y at w[k], w[as + k], w[2 as + k], w[3 as + k]; the two
// intermediates of each element go to v[2k], v[2k + 1].  FULL: a window
// after the first that ends before element m - 1 (tri_full_window), run
// without a condition per element -- lanes past the last system compute on
// the zeros their windows hold, and nothing reads their results -- so the
// window's loads issue ahead of the recurrence instead of one element at a
// time behind its branch.
__device__ __forceinline__ bool tri_full_window(int q, int m) { return q >= 1 && q * kTriWin + kTriWin < m; }
template <int FORM, bool FULL = false>
__device__ __forceinline__ void tri_forward_window(TriFwd& f, const float* w, int as, int q, int m, bool act,
                                                   float (&v)[16]) {
#pragma unroll
  for (int k = 0; k < kTriWin; k++) {
    const int i = q * kTriWin + k;
    v[2 * k] = 0.0f;
    v[2 * k + 1] = 0.0f;
    if (FULL || (act && i < m)) {
      const float ai = w[k], bi = w[as + k], ci = w[2 * as + k], yi = w[3 * as + k];
      if constexpr (FORM == 0) {
        // cp_i = c_i / (b_i - a_i cp_{i-1}), yp_i = (y_i - a_i yp_{i-1}) / (...)  (:82-91)
        if (!FULL && i == 0) {
          f.cp = tri_div(ci, bi);
          f.yp = tri_div(yi, bi);
        } else {
          const float nf = tri_rcp(tri_sub(bi, tri_mul(ai, f.cp)));
          f.cp = tri_mul(ci, nf);
          f.yp = tri_mul(tri_sub(yi, tri_mul(ai, f.yp)), nf);
        }
        v[2 * k] = f.cp;
        v[2 * k + 1] = f.yp;
      } else {
        // recurrence 1 (:9-33): b'_i from the 4-tuple scan of (b_i, -a_i c_{i-1}, 1, 0)
        if (!FULL && i == 0) {
          f.b0 = bi;
          f.y0 = yi;
        }
        float m0 = 1.0f, m1 = 0.0f, m2 = 0.0f, m3 = 1.0f;
        if (FULL || 0 < i) {
          m0 = bi;
          m1 = tri_sub(0.0f, tri_mul(ai, f.cprev));
          m2 = 1.0f;
          m3 = 0.0f;
        }
        f.cprev = ci;
        const float value = tri_rcp(tri_mul(f.s0, m0));
        const float n0 = tri_mul(tri_add(tri_mul(m0, f.s0), tri_mul(m1, f.s2)), value);
        const float n1 = tri_mul(tri_add(tri_mul(m0, f.s1), tri_mul(m1, f.s3)), value);
        const float n2 = tri_mul(tri_add(tri_mul(m2, f.s0), tri_mul(m3, f.s2)), value);
        const float n3 = tri_mul(tri_add(tri_mul(m2, f.s1), tri_mul(m3, f.s3)), value);
        f.s0 = n0;
        f.s1 = n1;
        f.s2 = n2;
        f.s3 = n3;
        const float bpi = tri_div(tri_add(tri_mul(f.s0, f.b0), f.s1), tri_add(tri_mul(f.s2, f.b0), f.s3));  // b'_i
        const double rbp = tri_rcpd(bpi);  // three quotients by b'_i: y'_i, c_i here, a_{i+1} next
        // recurrence 2 (:38-56): y'_i from the scan of (y_i, -a_i / b'_{i-1})
        float l0 = 0.0f, l1 = 1.0f;
        if (FULL || 0 < i) {
          l0 = yi;
          l1 = tri_sub(0.0f, tri_divr(ai, f.rbprev));
        }
        const float e0 = tri_add(l0, tri_mul(l1, f.c0));
        const float e1 = tri_mul(f.c1, l1);
        f.c0 = e0;
        f.c1 = e1;
        const float ypi = tri_add(f.c0, tri_mul(f.c1, f.y0));  // y'_i
        f.rbprev = rbp;
        // recurrence 3's elements (:61-79), the last one's first component
        // its starting value
        if (FULL || i < m - 1) {
          v[2 * k] = tri_divr(ypi, rbp);
          v[2 * k + 1] = tri_sub(0.0f, tri_divr(ci, rbp));
        } else {
          f.yn = tri_divr(ypi, rbp);
        }
      }
    }
  }
}

// The backward pass of a warp's nr systems (rows r0 ..), the intermediates
// read back from the warp's lane quarter of tensor memory (tl, column 0) a
// window at a time; the solution leaves through the output window Wo as
// 32-byte runs of rows.
template <int FORM>
__device__ __forceinline__ void tri_backward(TriFwd& f, uint32_t tl, float* Wo, int lane, int nr, int m, int64_t r0,
                                             float* __restrict__ out) {
  constexpr int WS = kTriWin + 1;
  const bool act = lane < nr;
  const int nq = (m + kTriWin - 1) / kTriWin;
  float x = f.yp;  // FORM 0: x_{m-1} = yp_{m-1}
  f.c0 = 0.0f;
  f.c1 = 1.0f;
  for (int q = nq - 1; q >= 0; q--) {
    float v[16];
    tmem_ld16(tl + 16 * q, v);
    const bool full = tri_full_window(q, m);  // no element of the window is past m - 2: no condition per element
#pragma unroll
    for (int k = kTriWin - 1; k >= 0; k--) {
      const int i = q * kTriWin + k;
      if (full || (act && i < m)) {
        if constexpr (FORM == 0) {
          // x_i = yp_i - cp_i x_{i+1}  (:92-95)
          if (full || i < m - 1) x = tri_sub(v[2 * k + 1], tri_mul(v[2 * k], x));
          Wo[lane * WS + k] = x;
        } else {
          float l0 = 0.0f, l1 = 1.0f;
          if (full || i < m - 1) {
            l0 = v[2 * k];
            l1 = v[2 * k + 1];
          }
          const float n0 = tri_add(l0, tri_mul(l1, f.c0));
          const float n1 = tri_mul(f.c1, l1);
          f.c0 = n0;
          f.c1 = n1;
          Wo[lane * WS + k] = tri_add(f.c0, tri_mul(f.c1, f.yn));
        }
      }
    }
    __syncwarp();
#pragma unroll
    for (int t = 0; t < kTriWin; t++) {
      const int idx = t * 32 + lane, row = idx / kTriWin, col = idx % kTriWin;
      const int gcol = q * kTriWin + col;
      if (row < nr && gcol < m) __stcs(out + (r0 + row) * (int64_t)m + gcol, Wo[row * WS + col]);
    }
    __syncwarp();  // the output window is rewritten next iteration
  }
}

template <int FORM, int COLS>
__global__ void __launch_bounds__(32 * kTriTmemWarps) lvc_tridag_tmem_kernel(int64_t rows, int m,
                                                                             const float* __restrict__ a,
                                                                             const float* __restrict__ b,
                                                                             const float* __restrict__ c,
                                                                             const float* __restrict__ y,
                                                                             float* __restrict__ out) {
  extern __shared__ __align__(16) unsigned char tri_raw[];
  constexpr int WS = kTriWin + 1, WA = 32 * WS, WB = 4 * WA;
  uint32_t* s_taddr = reinterpret_cast<uint32_t*>(tri_raw);  // written by tcgen05.alloc
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float* const Wn = reinterpret_cast<float*>(tri_raw + 16) + warp * (kTriTmemStages * WB + WA);  // input ring
  float* const Wo = Wn + kTriTmemStages * WB;                                                    // output window
  const int64_t r0 = ((int64_t)blockIdx.x * kTriTmemWarps + warp) * 32;
  // a warp past the last system still takes part in the CTA's allocation
  // and release of tensor memory
  const int nr = r0 < rows ? (int)(rows - r0 < 32 ? rows - r0 : 32) : 0;
  if (warp == 0) {
    tmem_alloc(s_taddr, COLS);
    tmem_relinquish();
  }
  tmem_fence_before_sync();
  __syncthreads();
  tmem_fence_after_sync();
  const uint32_t tl = *s_taddr + ((uint32_t)(32 * (warp & 3)) << 16);  // this warp's lane quarter, column 0
  if (nr > 0) {
    const float* src[4] = {a, b, c, y};
    const int nq = (m + kTriWin - 1) / kTriWin;
    const bool act = lane < nr;
    auto fetch = [&](int q) {
      if (q < nq) {
        float* const dst = Wn + (q % kTriTmemStages) * WB;
#pragma unroll
        for (int arr = 0; arr < 4; arr++) {
#pragma unroll
          for (int t = 0; t < kTriWin; t++) {
            const int idx = t * 32 + lane, row = idx / kTriWin, col = idx % kTriWin;
            const int gcol = q * kTriWin + col;
            const bool valid = row < nr && gcol < m;
            const float* g = valid ? src[arr] + (r0 + row) * (int64_t)m + gcol : src[arr];
            cp_async4(dst + arr * WA + row * WS + col, g, valid);
          }
        }
      }
      cp_async_commit();
    };
    TriFwd f;
    fetch(0);
    fetch(1);
    for (int q = 0; q < nq; q++) {
      fetch(q + 2);
      cp_async_wait<2>();  // window q has landed
      __syncwarp();
      float v[16];
      const float* const w = Wn + (q % kTriTmemStages) * WB + lane * WS;
      if (tri_full_window(q, m))
        tri_forward_window<FORM, true>(f, w, WA, q, m, act, v);
      else
        tri_forward_window<FORM>(f, w, WA, q, m, act, v);
      tmem_st16(tl + 16 * q, v);
      __syncwarp();  // this ring stage is refilled by the next iteration's fetch
    }
    cp_async_wait<0>();
    tmem_wait_st();
    tri_backward<FORM>(f, tl, Wo, lane, nr, m, r0, out);
  }
  tmem_fence_before_sync();
  __syncthreads();
  tmem_fence_after_sync();
  if (warp == 0) tmem_dealloc(*s_taddr, COLS);
}

// The same solver with the inputs staged by the tensor-memory accelerator
// (TMA) for the whole CTA, for odd m (up to kTriTmemMaxM) and rows % 4 == 0.
// Four consecutive systems of such a batch are one contiguous run of 4m
// floats whose start is 16-byte aligned (16m bytes apart), so each input is
// viewed as a 2-D tensor of rows / 4 "groups" of 4m floats.  Window q of
// system s of a group (elements 8q .. 8q + 7, at 4m-offset m s + 8q) lies
// inside the 12 floats from the 16-byte boundary at or below it, offset
// (m s) mod 4; one tensor copy per array and s brings that 12-float box of
// the CTA's 32 groups into shared memory -- and the box is 20 floats wide,
// so that it holds two windows (2j, 2j + 1: 16 elements from offset
// (m s) mod 4), [s][group][20]: sixteen copies per pair of windows for the
// CTA's 128 systems, against 32 four-byte cp.async per lane, array and
// window (boxes of one window, 12 floats, were 6 % slower: twice the box
// rows for the copy engine).  Lane l of warp w owns system
// 4 (8w + l / 4) + l % 4 and reads its elements at group 8w + l / 4 of box
// l % 4: with m odd the offsets (m s) mod 4 of the four boxes are distinct
// and 20 (8w + g) mod 32 runs over distinct multiples of 4, so a warp's
// reads are free of bank conflicts.  A fifth warp issues the copies into a
// ring of kTriTmaStages stages: window pair j lands on full[j % S]; each
// solving warp, done with a pair, arrives on empty[j % S], and the producer
// refills that stage with pair j + S once all four have -- so a solving
// warp waits only for its data, never for the other warps (a CTA barrier
// per window cost the solvers about a fifth of their time).  Every wait is
// bounded.  All four solving warps run the forward loop (the producer
// counts on their arrivals); warps past the last system compute on zeros
// and store nothing.
constexpr int kTriTmaBox = 20;                                        // floats per box row: two windows
constexpr int kTriTmaGroups = 8 * kTriTmemWarps;                      // 4-system groups per CTA
constexpr int kTriTmaStageFloats = 4 * 4 * kTriTmaGroups * kTriTmaBox;  // [array][s][group][box]
constexpr int kTriTmaStages = 2;
constexpr int kTriTmaThreads = 32 * (kTriTmemWarps + 1);                // four solving warps and the producer
__host__ __device__ __forceinline__ size_t tri_tma_smem(int cols) {
  const size_t need = 128 /* alignment */ + 128 /* barriers, TMEM address */ +
                      sizeof(float) * (kTriTmaStages * (size_t)kTriTmaStageFloats + kTriTmemWarps * 32 * (kTriWin + 1));
  // 87 KB: three CTAs never share an SM, so at most 512 TMEM columns are
  // asked for there; for 512-column CTAs, one per SM (as tri_tmem_smem)
  const size_t pad = cols > 256 ? 150 * 1024 : 0;
  return need > pad ? need : pad;
}
__device__ __forceinline__ void tma_load_2d(float* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n" ::"r"(
          smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

template <int FORM, int COLS>
__global__ void __launch_bounds__(kTriTmaThreads, 2) lvc_tridag_tma_kernel(const __grid_constant__ CUtensorMap ta,
                                                                       const __grid_constant__ CUtensorMap tb,
                                                                       const __grid_constant__ CUtensorMap tc,
                                                                       const __grid_constant__ CUtensorMap ty,
                                                                       int64_t rows, int m, float* __restrict__ out) {
  extern __shared__ __align__(16) unsigned char tri_raw[];
  constexpr int WS = kTriWin + 1, AS = 4 * kTriTmaGroups * kTriTmaBox, SS = kTriTmaGroups * kTriTmaBox;
  constexpr int S = kTriTmaStages;
  const uint32_t raw = smem_u32(tri_raw);
  unsigned char* const base = tri_raw + (((raw + 127u) & ~127u) - raw);  // 128-byte aligned
  uint64_t* const full = reinterpret_cast<uint64_t*>(base);                // [S]
  uint64_t* const empty = full + S;                                        // [S]
  uint32_t* const s_taddr = reinterpret_cast<uint32_t*>(base + 16 * S);    // written by tcgen05.alloc
  float* const stage0 = reinterpret_cast<float*>(base + 128);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g0 = blockIdx.x * kTriTmaGroups;  // the CTA's first group
  const int nq = (m + kTriWin - 1) / kTriWin;
  if (threadIdx.x == 0) {
    for (int i = 0; i < S; i++) {
      mbar_init(&full[i], 1);
      mbar_init(&empty[i], kTriTmemWarps);
    }
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 0) {
    tmem_alloc(s_taddr, COLS);
    tmem_relinquish();
  }
  tmem_fence_before_sync();
  __syncthreads();
  tmem_fence_after_sync();
  if (warp == kTriTmemWarps) {  // the producer
    if (lane == 0) {
      const int np = (nq + 1) / 2;
      for (int q = 0; q < np; q++) {
        const int st = q % S;
        if (q >= S && !mbar_wait(&empty[st], (unsigned)(q / S - 1) & 1u, kWaitPolls)) {
          atomicExch(&lvc_tridag_err, 1);  // the solvers' own waits then run out too
          break;
        }
        float* const dst = stage0 + st * kTriTmaStageFloats;
        mbar_expect_tx(&full[st], (unsigned)(sizeof(float) * kTriTmaStageFloats));
#pragma unroll
        for (int s = 0; s < 4; s++) {
          const int x = (m * s + 2 * kTriWin * q) & ~3;
          tma_load_2d(dst + s * SS, &ta, x, g0, &full[st]);
          tma_load_2d(dst + AS + s * SS, &tb, x, g0, &full[st]);
          tma_load_2d(dst + 2 * AS + s * SS, &tc, x, g0, &full[st]);
          tma_load_2d(dst + 3 * AS + s * SS, &ty, x, g0, &full[st]);
        }
      }
    }
  } else {
    float* const Wo = stage0 + S * kTriTmaStageFloats + warp * 32 * WS;  // output window
    const int64_t r0 = ((int64_t)blockIdx.x * kTriTmemWarps + warp) * 32;
    const int nr = r0 < rows ? (int)(rows - r0 < 32 ? rows - r0 : 32) : 0;
    const uint32_t tl = *s_taddr + ((uint32_t)(32 * (warp & 3)) << 16);  // this warp's lane quarter, column 0
    const int s = lane & 3;
    const float* const mine = stage0 + s * SS + (8 * warp + (lane >> 2)) * kTriTmaBox + ((m * s) & 3);
    const bool act = lane < nr;
    bool timed_out = false;
    TriFwd f;
    for (int q = 0; q < nq; q++) {
      const int j = q >> 1, st = j % S;
      if (!(q & 1) && !mbar_wait(&full[st], (unsigned)(j / S) & 1u, timed_out ? kWaitPollsAfterTimeout : kWaitPolls)) {
        timed_out = true;
        atomicExch(&lvc_tridag_err, 1);
      }
      float v[16];
      const float* const w = mine + st * kTriTmaStageFloats + kTriWin * (q & 1);
      if (tri_full_window(q, m))
        tri_forward_window<FORM, true>(f, w, AS, q, m, act, v);
      else
        tri_forward_window<FORM>(f, w, AS, q, m, act, v);
      tmem_st16(tl + 16 * q, v);
      __syncwarp();  // the whole warp has read the stage
      if (lane == 0 && ((q & 1) || q == nq - 1))
        asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(&empty[st])) : "memory");
    }
    if (timed_out && lane == 0) {  // copies that never landed: one more bounded wait for the last ones
      const int np = (nq + 1) / 2;
      for (int q = np > S ? np - S : 0; q < np; q++) mbar_wait(&full[q % S], (unsigned)(q / S) & 1u, kWaitPolls);
    }
    tmem_wait_st();
    if (nr > 0) tri_backward<FORM>(f, tl, Wo, lane, nr, m, r0, out);
  }
  tmem_fence_before_sync();
  __syncthreads();
  tmem_fence_after_sync();
  if (warp == 0) tmem_dealloc(*s_taddr, COLS);
}

}  // namespace lvc
