// The turbulent-kinetic-energy step of the ocean model,
// misc/ocean-sim/tke.fut (entry main, DTYPE = f32), behind the C API the
// Futhark compiler generates for that program (include/tke.h).  A library of
// its own: the program's entry point is named futhark_entry_main like
// LocVolCalib's.
//
// One step is three kernels on the context's stream:
//   tke_coef_kernel    delta and the tridiagonal coefficients a, b, c, d of
//                      every z column (tke.fut:103-210), one thread per cell;
//   lvc_tridag_block_kernel<1>  tridagPar along z (tke.fut:4-17, 211), the
//                      batched solver of lvc_tridiag.cuh with rows = xdim*ydim
//                      columns of length zdim;
//   tke_update_kernel  everything after the solve (tke.fut:212-347) for one
//                      cell: the water mask, the surface correction and the
//                      clip of the top cell, lateral diffusion, the advection
//                      fluxes east, north and top (recomputed at each
//                      neighbour rather than stored), dtketau and the
//                      Adams-Bashforth update.
// Every operation is explicitly rounded (no fused multiply-add) in the
// reference's operand order, so the outputs equal the CPU oracle's -- which
// reproduces the reference's golden outputs bit for bit -- exactly.  The work
// is a few tens of operations per cell over ~25 input arrays: HBM-bound.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <string>

#include "lvc_tridiag.cuh"
#include "tke.h"

using namespace lvc;

namespace {

__device__ __forceinline__ float M_(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float A_(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float S_(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float D_(float a, float b) { return __fdiv_rn(a, b); }
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
  float *a, *b, *c, *d, *sol;                                 // scratch [X][Y][Z]
  float *tketaup1_out, *dtketau_out, *tke_surf_corr_out;      // outputs
};

__device__ __forceinline__ int64_t i3(const TkeArgs& p, int x, int y, int z) {
  return ((int64_t)x * p.Y + y) * p.Z + z;
}
__device__ __forceinline__ bool interior(const TkeArgs& p, int x, int y) {
  return x >= 2 && x < p.X - 2 && y >= 2 && y < p.Y - 2;
}
// tke.fut:103-108
__device__ __forceinline__ float delta_at(const TkeArgs& p, int x, int y, int z) {
  if (!(interior(p, x, y) && z < p.Z - 1)) return 0.0f;
  return M_(M_(M_(D_(kDtTke, p.dzt[z + 1]), kAlphaTke), 0.5f),
            A_(p.kappaM[i3(p, x, y, z)], p.kappaM[i3(p, x, y, z + 1)]));
}

__global__ void __launch_bounds__(256) tke_coef_kernel(TkeArgs p) {
  const int64_t n = (int64_t)p.X * p.Y * p.Z;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int z = (int)(i % p.Z);
    const int64_t xy = i / p.Z;
    const int y = (int)(xy % p.Y), x = (int)(xy / p.Y);
    const float sqrttke = __fsqrt_rn(max_(0.0f, p.tketau[i]));
    float av = 0.0f, bv = 0.0f, cv = 0.0f, dv = 0.0f;
    if (interior(p, x, y)) {
      const int ks = p.kbot[xy] - 1;
      const bool land = ks >= 0, edge = land && z == ks, water = land && z >= ks;
      const float dz = p.dzw[z];
      const float d0 = delta_at(p, x, y, z);
      const float dm = z > 0 ? delta_at(p, x, y, z - 1) : 0.0f;
      // a_tri (:109-122)
      if (edge || !water) av = 0.0f;
      else if (z > 0 && z < p.Z - 1) av = D_(-dm, dz);
      else if (z == p.Z - 1) av = D_(-dm, M_(0.5f, dz));
      // b_tri (:123-146)
      if (!water) bv = 1.0f;
      else if (edge) bv = A_(A_(1.0f, D_(d0, dz)), M_(D_(M_(kDtTke, kCEps), p.mxl[i]), sqrttke));
      else if (z > 0 && z < p.Z - 1) bv = A_(A_(1.0f, D_(A_(d0, dm), dz)), D_(M_(M_(kDtTke, kCEps), sqrttke), p.mxl[i]));
      else if (z == p.Z - 1) bv = A_(A_(1.0f, D_(dm, M_(0.5f, dz))), M_(D_(M_(kDtTke, kCEps), p.mxl[i]), sqrttke));
      // c_tri (:187-196)
      if (z < p.Z - 1) cv = water ? D_(-d0, dz) : 0.0f;
      // d_tri (:197-210)
      if (water) {
        const float tmp = A_(p.tketau[i], M_(kDtTke, p.forc[i]));
        dv = (z == p.Z - 1) ? A_(tmp, D_(M_(kDtTke, p.forc_tke_surface[xy]), M_(0.5f, dz))) : tmp;
      }
    }
    p.a[i] = av;
    p.b[i] = bv;
    p.c[i] = cv;
    p.d[i] = dv;
  }
}

// tke.fut:19-41
__device__ __forceinline__ float limiter(float cr) {
  return max_(0.0f, max_(min_(1.0f, M_(2.0f, cr)), min_(2.0f, cr)));
}
__device__ __forceinline__ float calcflux(float velfac, float velS, float dt_tracer, float dx, float varS,
                                          float varSM1, float varSP1, float varSP2, float maskS, float maskSM1,
                                          float maskSP1) {
  const float scaledVel = M_(velfac, velS);
  const float uCFL = fabsf(D_(M_(scaledVel, dt_tracer), dx));
  const float rjp = M_(S_(varSP2, varSP1), maskSP1);
  const float rj = M_(S_(varSP1, varS), maskS);
  const float rjm = M_(S_(varS, varSM1), maskSM1);
  const float epsilon = 0.00000000000000000001f;
  const float divisor = (fabsf(rj) < epsilon) ? epsilon : rj;
  float cr = (velS > 0.0f) ? D_(rjm, divisor) : D_(rjp, divisor);
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
  return calcflux(1.0f, p.utau[i], kDtTracer, dx, p.tketau[i], p.tketau[i3(p, x - 1, y, z)],
                  p.tketau[i3(p, x + 1, y, z)], p.tketau[i3(p, x + 2, y, z)], in ? M_(mWs, mWp1) : 0.0f,
                  in ? M_(mWm1, mWs) : 0.0f, in ? M_(mWp1, mWp2) : 0.0f);
}
__device__ __forceinline__ float adv_north(const TkeArgs& p, int x, int y, int z) {
  if (!(y >= 1 && y < p.Y - 2 && x >= 2 && x < p.X - 2)) return 0.0f;
  const int64_t i = i3(p, x, y, z);
  const float dx = M_(p.cost[y], p.dyt[y]);
  const float mWm1 = p.maskW[i3(p, x, y - 1, z)], mWs = p.maskW[i], mWp1 = p.maskW[i3(p, x, y + 1, z)],
              mWp2 = p.maskW[i3(p, x, y + 2, z)];
  const bool in = y < p.Y - 1;
  return calcflux(p.cosu[y], p.vtau[i], kDtTracer, dx, p.tketau[i], p.tketau[i3(p, x, y - 1, z)],
                  p.tketau[i3(p, x, y + 1, z)], p.tketau[i3(p, x, y + 2, z)], in ? M_(mWs, mWp1) : 0.0f,
                  in ? M_(mWm1, mWs) : 0.0f, in ? M_(mWp1, mWp2) : 0.0f);
}
__device__ __forceinline__ float adv_top(const TkeArgs& p, int x, int y, int z) {
  if (!(z < p.Z - 1 && interior(p, x, y))) return 0.0f;
  const int64_t i = i3(p, x, y, z);
  const float varSM1 = z != 0 ? p.tketau[i - 1] : 0.0f;
  const float varSP2 = z < p.Z - 2 ? p.tketau[i + 2] : 0.0f;
  const float mWm1 = z != 0 ? p.maskW[i - 1] : 0.0f;
  const float mWs = p.maskW[i], mWp1 = p.maskW[i + 1];
  const float mWp2 = z < p.Z - 2 ? p.maskW[i + 2] : 0.0f;
  return calcflux(1.0f, p.wtau[i], kDtTracer, p.dzw[z], p.tketau[i], varSM1, p.tketau[i + 1], varSP2,
                  M_(mWs, mWp1), M_(mWm1, mWs), M_(mWp1, mWp2));
}

__global__ void __launch_bounds__(256) tke_update_kernel(TkeArgs p) {
  const int64_t n = (int64_t)p.X * p.Y * p.Z;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int z = (int)(i % p.Z);
    const int64_t xy = i / p.Z;
    const int y = (int)(xy % p.Y), x = (int)(xy / p.Y);
    const bool inner = interior(p, x, y);
    const int ks = p.kbot[xy] - 1;
    const bool water = ks >= 0 && z >= ks;
    float tp = (inner && water) ? p.sol[i] : p.tketaup1[i];  // :212-218
    if (z == p.Z - 1) {
      // surface correction (:219-226), from the value before the clip
      float corr = 0.0f;
      if (inner && tp < 0.0f) corr = D_(M_(M_(-tp, 0.5f), p.dzw[p.Z - 1]), kDtTke);
      p.tke_surf_corr_out[xy] = corr;
      if (inner) {
        tp = tp < 0.0f ? 0.0f : tp;  // :227-235
        // lateral diffusion (:252-263)
        tp = A_(tp, M_(M_(kDtTke, p.maskW[i]),
                       A_(D_(S_(diff_east(p, x, y, z), diff_east(p, x - 1, y, z)), M_(p.cost[y], p.dxt[x])),
                          D_(S_(diff_north(p, x, y, z), diff_north(p, x, y - 1, z)), M_(p.cost[y], p.dyt[y])))));
      }
    }
    // dtketau (:320-340)
    float tmp = p.dtketau[i];
    if (inner)
      tmp = M_(p.maskW[i], S_(D_(-S_(adv_east(p, x, y, z), adv_east(p, x - 1, y, z)), M_(p.cost[y], p.dxt[x])),
                              D_(S_(adv_north(p, x, y, z), adv_north(p, x, y - 1, z)), M_(p.cost[y], p.dyt[y]))));
    const float ft = adv_top(p, x, y, z);
    const float ftm = z >= 1 ? adv_top(p, x, y, z - 1) : 0.0f;
    const float z0 = z == 0 ? S_(tmp, D_(ft, p.dzw[0])) : tmp;
    const float zm = (z >= 1 && z < p.Z - 1) ? S_(z0, D_(S_(ft, ftm), p.dzw[z])) : z0;
    const float dtk = (z == p.Z - 1) ? S_(zm, D_(S_(ft, ftm), M_(0.5f, p.dzw[z]))) : zm;
    p.dtketau_out[i] = dtk;
    // Adams-Bashforth (:341-347)
    p.tketaup1_out[i] =
        A_(tp, M_(kDtTracer, S_(M_(A_(1.5f, kABEps), dtk), M_(A_(0.5f, kABEps), p.dtketaum1[i]))));
  }
}

}  // namespace

// ---------------------------------------------------------------------------
// Contexts and arrays (the generated API's shapes)
// ---------------------------------------------------------------------------
struct futhark_context_config {
  int device = 0;
};
struct futhark_context {
  std::mutex mu;
  int device = 0;
  int num_sms = 0;
  cudaStream_t stream = nullptr;
  std::string error;
  bool ok = false;
  void* scratch = nullptr;  // the entry point's step scratch, grown on demand
  size_t scratch_bytes = 0;
};

namespace {

// Device storage shared by the arrays that view it: the entry point returns
// its four pass-through outputs as views of the consumed inputs' storage.
struct DevMem {
  void* p = nullptr;
  int refs = 1;
};

}  // namespace

template <typename T, int R>
struct DevArray {
  T* data = nullptr;
  DevMem* mem = nullptr;
  int64_t shape[R] = {};
  int64_t n() const {
    int64_t k = 1;
    for (int r = 0; r < R; r++) k *= shape[r];
    return k;
  }
};
struct futhark_f32_1d : DevArray<float, 1> {};
struct futhark_f32_2d : DevArray<float, 2> {};
struct futhark_f32_3d : DevArray<float, 3> {};
struct futhark_i32_2d : DevArray<int32_t, 2> {};

namespace {

int set_error(futhark_context* ctx, int code, const std::string& msg) {
  ctx->error = msg;
  return code;
}
int cuda_fail(futhark_context* ctx, cudaError_t e, const char* what) {
  return set_error(ctx, e == cudaErrorMemoryAllocation ? FUTHARK_OUT_OF_MEMORY : FUTHARK_PROGRAM_ERROR,
                   std::string(what) + ": " + cudaGetErrorString(e));
}

void release(DevMem* m) {
  if (m && --m->refs == 0) {
    cudaFree(m->p);
    delete m;
  }
}

template <typename A>
A* alloc_array(const int64_t* dims, int rank) {
  auto* a = new (std::nothrow) A();
  if (!a) return nullptr;
  for (int r = 0; r < rank; r++) a->shape[r] = dims[r];
  a->mem = new (std::nothrow) DevMem();
  if (!a->mem ||
      cudaMalloc(&a->mem->p, sizeof(*a->data) * (size_t)std::max<int64_t>(1, a->n())) != cudaSuccess) {
    cudaGetLastError();
    delete a->mem;
    delete a;
    return nullptr;
  }
  a->data = static_cast<decltype(a->data)>(a->mem->p);
  return a;
}
template <typename A>
void drop_array(A* a) {
  if (!a) return;
  release(a->mem);
  delete a;
}

template <typename A, typename T>
A* new_array(futhark_context* ctx, const T* data, const int64_t* dims, int rank) {
  std::lock_guard<std::mutex> g(ctx->mu);
  if (!ctx->ok) {
    ctx->error = "context has no usable CUDA device";
    return nullptr;
  }
  for (int r = 0; r < rank; r++)
    if (dims[r] < 0) {
      ctx->error = "negative array dimension";
      return nullptr;
    }
  cudaSetDevice(ctx->device);
  A* a = alloc_array<A>(dims, rank);
  if (!a) {
    ctx->error = "out of device memory";
    return nullptr;
  }
  if (a->n() > 0 && data) {
    cudaError_t e = cudaMemcpyAsync(a->data, data, sizeof(T) * a->n(), cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
      drop_array(a);
      cuda_fail(ctx, e, "host to device copy");
      return nullptr;
    }
  }
  return a;
}
template <typename A>
int free_array(futhark_context* ctx, A* a) {
  if (!a) return 0;
  std::lock_guard<std::mutex> g(ctx->mu);
  if (ctx->ok) {
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);  // no launch still reads it
  }
  drop_array(a);
  return 0;
}
template <typename A, typename T>
int values_array(futhark_context* ctx, A* a, T* out) {
  std::lock_guard<std::mutex> g(ctx->mu);
  if (!ctx->ok) return set_error(ctx, FUTHARK_PROGRAM_ERROR, "context has no usable CUDA device");
  if (!a || (!out && a->n() > 0)) return set_error(ctx, FUTHARK_PROGRAM_ERROR, "null array");
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e == cudaSuccess && a->n() > 0)
    e = cudaMemcpyAsync(out, a->data, sizeof(T) * a->n(), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  return e == cudaSuccess ? 0 : cuda_fail(ctx, e, "device to host copy");
}

size_t scratch_bytes(int64_t X, int64_t Y, int64_t Z) {
  // a, b, c, d, sol and the generic solver's pivots (zdim > kTriBlockMaxM),
  // each on a 128-byte boundary for the block solver's bulk copies
  const int64_t ns = (X * Y * Z + 31) & ~int64_t(31);
  return 6 * sizeof(float) * (size_t)std::max<int64_t>(32, ns);
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
  const int64_t ns = (n + 31) & ~int64_t(31);
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
  p.a = scratch;
  p.b = scratch + ns;
  p.c = scratch + 2 * ns;
  p.d = scratch + 3 * ns;
  p.sol = scratch + 4 * ns;
  p.tketaup1_out = q->tketaup1_out;
  p.dtketau_out = q->dtketau_out;
  p.tke_surf_corr_out = q->tke_surf_corr_out;
  cudaStream_t s = ctx->stream;
  const int grid = (int)std::min<int64_t>((n + 255) / 256, 32LL * ctx->num_sms);
  tke_coef_kernel<<<grid, 256, 0, s>>>(p);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(ctx, e, "tke coefficient launch");
  // the vertical solve: X*Y systems of length Z (tke.fut:4-17, 211)
  const int64_t rows = X * Y;
  if (Z <= kTriBlockMaxM) {
    const size_t bs = (size_t)((kTriBlockRows * Z + 3) & ~int64_t(3));
    const size_t smem = 16 + 4 * bs * sizeof(float);
    const size_t smem_max = 16 + 4 * (size_t)((kTriBlockRows * kTriBlockMaxM + 3) & ~3) * sizeof(float);
    e = cudaFuncSetAttribute((const void*)lvc_tridag_block_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem_max);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "tke solver attributes");
    lvc_tridag_block_kernel<1><<<(unsigned)((rows + kTriBlockRows - 1) / kTriBlockRows), kTriBlockRows, smem, s>>>(
        rows, (int)Z, p.a, p.b, p.c, p.d, p.sol, 1);
  } else {
    lvc_tridag_kernel<1><<<(unsigned)((rows + kTriThreads - 1) / kTriThreads), kTriThreads, 0, s>>>(
        rows, (int)Z, p.a, p.b, p.c, p.d, p.sol, scratch + 5 * ns);
  }
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(ctx, e, "tke solver launch");
  tke_update_kernel<<<grid, 256, 0, s>>>(p);
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(ctx, e, "tke update launch");
  return 0;
}

// Synchronises and reads (then clears) the solver's timeout flag (lock held).
int check_locked(futhark_context* ctx) {
  int flag = 0;
  const int zero = 0;
  cudaError_t e = cudaMemcpyFromSymbolAsync(&flag, lvc_tridag_err, sizeof flag, 0, cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaMemcpyToSymbolAsync(lvc_tridag_err, &zero, sizeof zero, 0, cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "tke step");
  if (flag) return set_error(ctx, FUTHARK_PROGRAM_ERROR, "tke step: the vertical solve gave up waiting on a copy");
  return 0;
}

}  // namespace

extern "C" {

struct futhark_context_config* futhark_context_config_new(void) {
  return new (std::nothrow) futhark_context_config();
}
void futhark_context_config_free(struct futhark_context_config* cfg) { delete cfg; }
void futhark_context_config_set_device(struct futhark_context_config* cfg, const char* s) {
  if (cfg && s && s[0] == '#') cfg->device = atoi(s + 1);
}
void futhark_context_config_set_debugging(struct futhark_context_config*, int) {}
void futhark_context_config_set_profiling(struct futhark_context_config*, int) {}
void futhark_context_config_set_logging(struct futhark_context_config*, int) {}

struct futhark_context* futhark_context_new(struct futhark_context_config* cfg) {
  auto* ctx = new (std::nothrow) futhark_context();
  if (!ctx) return nullptr;
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  const int dev = cfg ? cfg->device : 0;
  if (e != cudaSuccess || ndev == 0 || dev < 0 || dev >= ndev) {
    cudaGetLastError();
    ctx->error = std::string("no usable CUDA device: ") + cudaGetErrorString(e);
    return ctx;
  }
  cudaDeviceProp prop;
  if ((e = cudaSetDevice(dev)) != cudaSuccess || (e = cudaGetDeviceProperties(&prop, dev)) != cudaSuccess) {
    ctx->error = std::string("cannot use CUDA device: ") + cudaGetErrorString(e);
    return ctx;
  }
  if (prop.major < 10) {
    ctx->error = "this build targets sm_100a (Blackwell)";
    return ctx;
  }
  if ((e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking)) != cudaSuccess) {
    ctx->error = std::string("cannot create a stream: ") + cudaGetErrorString(e);
    return ctx;
  }
  ctx->device = dev;
  ctx->num_sms = prop.multiProcessorCount;
  ctx->ok = true;
  return ctx;
}
void futhark_context_free(struct futhark_context* ctx) {
  if (!ctx) return;
  if (ctx->ok) {
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    if (ctx->scratch) cudaFree(ctx->scratch);
    cudaStreamDestroy(ctx->stream);
  }
  delete ctx;
}
int futhark_context_sync(struct futhark_context* ctx) {
  std::lock_guard<std::mutex> g(ctx->mu);
  if (!ctx->ok) return set_error(ctx, FUTHARK_PROGRAM_ERROR, "context has no usable CUDA device");
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  return e == cudaSuccess ? 0 : cuda_fail(ctx, e, "sync");
}
char* futhark_context_get_error(struct futhark_context* ctx) {
  std::lock_guard<std::mutex> g(ctx->mu);
  if (ctx->error.empty()) return nullptr;
  char* s = (char*)malloc(ctx->error.size() + 1);
  if (s) memcpy(s, ctx->error.c_str(), ctx->error.size() + 1);
  ctx->error.clear();
  return s;
}
int futhark_context_clear_caches(struct futhark_context* ctx) {
  std::lock_guard<std::mutex> g(ctx->mu);
  if (!ctx->ok) return 0;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  if (ctx->scratch) cudaFree(ctx->scratch);
  ctx->scratch = nullptr;
  ctx->scratch_bytes = 0;
  return 0;
}

#define TKE_ARRAY_API(NAME, T, R, ...)                                                                 \
  struct futhark_##NAME* futhark_new_##NAME(struct futhark_context* ctx, const T* data, __VA_ARGS__) { \
    const int64_t dims[] = {TKE_DIMS_##R};                                                             \
    return new_array<futhark_##NAME, T>(ctx, data, dims, R);                                           \
  }                                                                                                    \
  int futhark_free_##NAME(struct futhark_context* ctx, struct futhark_##NAME* arr) {                   \
    return free_array(ctx, arr);                                                                       \
  }                                                                                                    \
  int futhark_values_##NAME(struct futhark_context* ctx, struct futhark_##NAME* arr, T* data) {        \
    return values_array<futhark_##NAME, T>(ctx, arr, data);                                            \
  }                                                                                                    \
  const int64_t* futhark_shape_##NAME(struct futhark_context* ctx, struct futhark_##NAME* arr) {       \
    (void)ctx;                                                                                         \
    return arr ? arr->shape : nullptr;                                                                 \
  }
#define TKE_DIMS_1 dim0
#define TKE_DIMS_2 dim0, dim1
#define TKE_DIMS_3 dim0, dim1, dim2
TKE_ARRAY_API(f32_1d, float, 1, int64_t dim0)
TKE_ARRAY_API(f32_2d, float, 2, int64_t dim0, int64_t dim1)
TKE_ARRAY_API(f32_3d, float, 3, int64_t dim0, int64_t dim1, int64_t dim2)
TKE_ARRAY_API(i32_2d, int32_t, 2, int64_t dim0, int64_t dim1)

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
  const size_t need = scratch_bytes(X, Y, Z);
  if (up1 && dtk && corr && ctx->scratch_bytes < need) {
    cudaStreamSynchronize(ctx->stream);
    if (ctx->scratch) cudaFree(ctx->scratch);
    ctx->scratch = nullptr;
    ctx->scratch_bytes = 0;
    if (cudaMalloc(&ctx->scratch, need) == cudaSuccess) ctx->scratch_bytes = need;
    else cudaGetLastError();
  }
  if (!up1 || !dtk || !corr || ctx->scratch_bytes < need) {
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
