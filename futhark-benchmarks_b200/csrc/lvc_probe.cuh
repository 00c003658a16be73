// Peak probes: the two ceilings of the rollback kernel, measured on the
// device it runs on (the path is bound by the FP64 pipe and by shared-memory
// bandwidth, neither of which a copy or GEMM benchmark measures).
//
//   lvc_probe_dfma_kernel  8 independent FMA chains per thread, all SMs busy;
//                          2 flops per DFMA.
//   lvc_probe_smem_kernel  conflict-free 16-byte shared-memory loads by every
//                          thread, 4 independent loads per iteration.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace lvc {

constexpr int kProbeChains = 8;

__global__ void __launch_bounds__(256) lvc_probe_dfma_kernel(double* out, int iters, double b,
                                                             double c) {
  double a[kProbeChains];
#pragma unroll
  for (int k = 0; k < kProbeChains; k++) a[k] = 1e-3 * (threadIdx.x + k);
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int k = 0; k < kProbeChains; k++) a[k] = fma(a[k], b, c);
  }
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < kProbeChains; k++) s += a[k];
  if (s == 12345.678) out[blockIdx.x] = s;  // keeps the chains alive
}

constexpr int kProbeSmemVec = 2048;  // double2 elements = 32 KiB (static limit is 48 KiB)

__global__ void __launch_bounds__(512) lvc_probe_smem_kernel(unsigned long long* out, int iters) {
  __shared__ double2 buf[kProbeSmemVec];
  for (int i = threadIdx.x; i < kProbeSmemVec; i += blockDim.x)
    buf[i] = make_double2((double)i, (double)(i ^ 7));
  __syncthreads();
  unsigned long long acc = 0;
  const int lane_base = threadIdx.x;
  for (int i = 0; i < iters; i++) {
    const int o = (i * 64) & (kProbeSmemVec - 1);
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const double2 v = buf[(lane_base + o + k * 512) & (kProbeSmemVec - 1)];
      acc ^= (unsigned long long)__double_as_longlong(v.x) + (unsigned long long)__double_as_longlong(v.y);
    }
  }
  if (acc == 0x123456789ull) out[blockIdx.x] = acc;
}

}  // namespace lvc
