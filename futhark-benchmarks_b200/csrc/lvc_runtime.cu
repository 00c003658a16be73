// Host runtime of the LocVolCalib engine: contexts, batch plans (device
// tables, work lists, launch classes, captured CUDA graph) and the C API
// declared in include/LocVolCalib.h.
//
// A plan is built once per list of calibrations:
//   * every calibration gets an operator-table block and an X-pivot block in
//     two HBM arenas, and a price range in the output vector;
//   * every strike instance becomes a work item; items are grouped into launch
//     classes by kernel configuration (threads per CTA, lane chunk width,
//     cluster size, on-chip or HBM grid) and sorted by descending work
//     (longest-processing-time first) inside a class;
//   * one run = setup kernel + pivot kernel + one persistent rollback launch
//     per class, captured once into a CUDA graph.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "LocVolCalib.h"
#include "lvc_kernels.cuh"
#include "lvc_line.cuh"
#include "lvc_probe.cuh"

using namespace lvc;

struct futhark_context_config {
  int device = 0;
  std::string device_name;
  int debugging = 0, profiling = 0, logging = 0;
};

struct futhark_f32_1d {
  float* data;
  int64_t shape[1];
  size_t bytes;
};
struct futhark_f64_1d {
  double* data;
  int64_t shape[1];
  size_t bytes;
};

namespace {

struct Launch {
  int kind, NT, KX, C;
  bool gstate;
  bool full = false;
  int item_off, n_items, grid;
  size_t smem_bytes;
  int64_t gstate_per_cta;  // elements of the state type
  int64_t gstate_off;      // elements
};

}  // namespace

struct lvc_plan {
  int precision = LVC_F64;
  int ncal = 0;
  int64_t nprices = 0;
  std::vector<lvc_calibration> params;
  std::vector<CalibDev> calibs;
  std::vector<Launch> launches;
  std::vector<Item> items;
  std::vector<int64_t> row_start;
  int64_t tab_elems = 0, piv_elems = 0, gstate_elems = 0;
  CalibDev* d_calibs = nullptr;
  double* d_tabs = nullptr;
  void* d_piv = nullptr;
  double* d_out = nullptr;
  int64_t* d_rowstart = nullptr;
  Item* d_items = nullptr;
  void* d_gstate = nullptr;
  int* d_err = nullptr;
  int pivot_grid = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  double rollback_ms = 0.0;
};

struct futhark_context {
  std::mutex mu;
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t capture = nullptr;
  std::string error;
  int num_sms = 0;
  int max_smem = 0;
  bool ok = false;
  lvc_plan* entry_plan = nullptr;  // reused by the entry points while sizes repeat
};

namespace {

int set_error(futhark_context* ctx, int code, const std::string& msg) {
  ctx->error = msg;
  return code;
}

int cuda_fail(futhark_context* ctx, cudaError_t e, const char* what) {
  std::string msg = std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e);
  return set_error(ctx, e == cudaErrorMemoryAllocation ? FUTHARK_OUT_OF_MEMORY : FUTHARK_PROGRAM_ERROR,
                   msg);
}

#define LVC_CUDA(ctx, call)                                \
  do {                                                     \
    cudaError_t e_ = (call);                               \
    if (e_ != cudaSuccess) return cuda_fail(ctx, e_, #call); \
  } while (0)

int pow2ceil(int v) {
  int p = 1;
  while (p < v) p <<= 1;
  return p;
}

// Host restatement of initGrid's spot index (:16-20), same IEEE f64 operations
// as the setup kernel.  Returns false when the reference would index out of
// bounds at :236.
bool spot_index(double s0, double alpha, double t, int numX, int* xi) {
  const double stdX = 20.0 * alpha * s0 * std::sqrt(t);
  const double dx = stdX / (double)numX;
  const double v = s0 / dx;
  if (!(v >= 0.0) || !(v < (double)numX)) return false;
  *xi = (int)v;
  return true;
}

int validate(futhark_context* ctx, const lvc_calibration& c, int idx) {
  char buf[256];
  if (c.outer < 0 || c.numX < 3 || c.numY < 3 || c.numT < 1) {
    snprintf(buf, sizeof buf,
             "calibration %d: invalid sizes outer=%d numX=%d numY=%d numT=%d (need outer >= 0, "
             "numX >= 3, numY >= 3, numT >= 1)",
             idx, c.outer, c.numX, c.numY, c.numT);
    return set_error(ctx, FUTHARK_PROGRAM_ERROR, buf);
  }
  if (c.numX > 512 || c.numY > 1024) {
    snprintf(buf, sizeof buf,
             "calibration %d: numX=%d numY=%d beyond the engine's limits (numX <= 512, "
             "numY <= 1024)",
             idx, c.numX, c.numY);
    return set_error(ctx, FUTHARK_PROGRAM_ERROR, buf);
  }
  int xi;
  if (!spot_index(c.s0, c.alpha, c.t, c.numX, &xi)) {
    snprintf(buf, sizeof buf,
             "calibration %d: spot index s0/dx of initGrid lies outside [0, numX=%d); the "
             "reference program fails its bounds check here",
             idx, c.numX);
    return set_error(ctx, FUTHARK_PROGRAM_ERROR, buf);
  }
  return 0;
}

template <typename S, typename PV>
using RbFn = void (*)(RollbackArgs<S, PV>);

template <typename S, typename PV>
RbFn<S, PV> rollback_fn(int kind, int NT, int KX, bool gs, bool full = false) {
  if (kind == kKindLine && full) {
    if (NT == 32) return lvc_line_full_kernel<S, PV, 32, 2>;
    if (NT == 64) return lvc_line_full_kernel<S, PV, 64, 2>;
    if (NT == 128) return lvc_line_full_kernel<S, PV, 128, 2>;
    if (NT == 256) return lvc_line_full_kernel<S, PV, 256, 2>;
    return nullptr;
  }
  if (kind == kKindLine) {
    if (NT == 64) return lvc_line_kernel<S, PV, 64>;
    if (NT == 128) return lvc_line_kernel<S, PV, 128>;
    if (NT == 256) return lvc_line_kernel<S, PV, 256>;
    if (NT == 512) return lvc_line_kernel<S, PV, 512>;
    return nullptr;
  }
#define LVC_CASE(nt, kx, g) \
  if (NT == nt && KX == kx && gs == g) return lvc_rollback_kernel<S, PV, nt, kx, g>;
  LVC_CASE(128, 8, false)
  LVC_CASE(256, 8, false)
  LVC_CASE(512, 8, false)
  LVC_CASE(128, 16, false)
  LVC_CASE(256, 16, false)
  LVC_CASE(128, 8, true)
  LVC_CASE(256, 8, true)
  LVC_CASE(512, 8, true)
  LVC_CASE(128, 16, true)
  LVC_CASE(256, 16, true)
#undef LVC_CASE
  return nullptr;
}

template <typename S>
int state_size() { return (int)sizeof(S); }

// Kernel configuration of one calibration.
struct Config {
  int kind, NT, KX, C;
  bool gstate;
  bool full = false;
  int Ycs;
  size_t smem_bytes;
  int64_t grid_elems;
};

// Line family: one lane per grid line; needs numX <= 256 and at most 16
// warps of units per CTA, which fixes the cluster size.
template <typename S>
bool choose_line(int X, int Y, int max_smem, Config& cf) {
  if (X > 256) return false;
  for (int C = 1; C <= kMaxCluster; C *= 2) {
    // full tiles: every line chunk, row group and CTA block complete; two
    // units per warp, one unit per 512 cells
    if (X % 32 == 0 && Y % C == 0 && (Y / C) % 32 == 0) {
      const int Ycs = Y / C;
      const int units = X * Ycs / 512;
      const FullLayout F = full_layout<S>(X, Ycs, units);
      if (units >= 2 && units <= 16 && F.Ux == units && F.Uy == units && F.total <= max_smem) {
        cf.kind = kKindLine;
        cf.full = true;
        cf.NT = 16 * units;  // 32 lanes x units / 2 units per warp
        cf.KX = kLineK;
        cf.C = C;
        cf.gstate = false;
        cf.Ycs = Ycs;
        cf.smem_bytes = (size_t)F.total;
        cf.grid_elems = 0;
        return true;
      }
    }
    // rows per CTA: a multiple of 4 when split, so every CTA's bulk copies
    // start on a 16-byte boundary
    const int Ycs = C == 1 ? Y : (int)round4(ceil_div(Y, C));
    if (C > 1 && (C - 1) * Ycs >= Y) break;
    const LineLayout L16 = line_layout<S>(X, Ycs, 16);
    if (L16.Ux > 16 || L16.Uy > 16) continue;
    const int NT = std::max(64, 32 * pow2ceil(std::max(L16.Ux, L16.Uy)));
    const LineLayout L = line_layout<S>(X, Ycs, NT / 32);
    if (L.total > max_smem) continue;
    cf.kind = kKindLine;
    cf.full = false;
    cf.NT = NT;
    cf.KX = kLineK;
    cf.C = C;
    cf.gstate = false;
    cf.Ycs = Ycs;
    cf.smem_bytes = (size_t)L.total;
    cf.grid_elems = 0;
    return true;
  }
  return false;
}

template <typename S>
Config choose_config(int X, int Y, int max_smem) {
  Config cf;
  if (choose_line<S>(X, Y, max_smem, cf)) return cf;
  cf.kind = kKindChunk;
  const int Xp = std::max(8, pow2ceil(X));
  cf.KX = Xp <= 256 ? 8 : 16;
  cf.gstate = true;
  cf.C = 1;
  cf.Ycs = Y;
  for (int C = 1; C <= kMaxCluster; C *= 2) {
    const int Ycs = ceil_div(Y, C);
    if (C > 1 && (C - 1) * Ycs >= Y) break;  // a CTA would own no row
    const SmemLayout L = smem_layout<S>(Xp, X, Ycs, true);
    if ((size_t)L.total * sizeof(S) <= (size_t)max_smem) {
      cf.C = C;
      cf.Ycs = Ycs;
      cf.gstate = false;
      break;
    }
  }
  const SmemLayout L = smem_layout<S>(Xp, X, cf.Ycs, !cf.gstate);
  cf.smem_bytes = (size_t)L.total * sizeof(S);
  cf.grid_elems = L.grid_elems;
  const int cells = cf.Ycs * Xp;
  cf.NT = cells >= 4096 ? 512 : (cells >= 1024 ? 256 : 128);
  if (cf.KX == 16) cf.NT = std::min(cf.NT, 256);
  return cf;
}

template <typename S, typename PV>
int prepare_launch(futhark_context* ctx, Launch& L) {
  RbFn<S, PV> fn = rollback_fn<S, PV>(L.kind, L.NT, L.KX, L.gstate, L.full);
  if (!fn) return set_error(ctx, FUTHARK_PROGRAM_ERROR, "no rollback kernel for this configuration");
  // Several launch classes may share one kernel instantiation with different
  // shared-memory sizes: allow the device maximum once for all of them.
  LVC_CUDA(ctx, cudaFuncSetAttribute((const void*)fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     ctx->max_smem));
  if (L.C > 8)
    LVC_CUDA(ctx, cudaFuncSetAttribute((const void*)fn,
                                       cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
  int resident = 0;
  if (L.C == 1) {
    int per_sm = 0;
    LVC_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, L.NT, L.smem_bytes));
    resident = per_sm * ctx->num_sms;
  } else {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(L.C * std::max(1, L.n_items));
    cfg.blockDim = dim3(L.NT);
    cfg.dynamicSmemBytes = L.smem_bytes;
    cudaLaunchAttribute attr;
    attr.id = cudaLaunchAttributeClusterDimension;
    attr.val.clusterDim.x = L.C;
    attr.val.clusterDim.y = 1;
    attr.val.clusterDim.z = 1;
    cfg.attrs = &attr;
    cfg.numAttrs = 1;
    int ncl = 0;
    LVC_CUDA(ctx, cudaOccupancyMaxActiveClusters(&ncl, fn, &cfg));
    resident = ncl;
  }
  if (resident <= 0)
    return set_error(ctx, FUTHARK_PROGRAM_ERROR, "rollback configuration does not fit on the device");
  L.grid = std::min(L.n_items, resident) * L.C;
  return 0;
}

template <typename S, typename PV>
cudaError_t launch_rollback(lvc_plan* P, const Launch& L, cudaStream_t s) {
  RollbackArgs<S, PV> a;
  a.calibs = P->d_calibs;
  a.items = P->d_items + L.item_off;
  a.n_items = L.n_items;
  a.C = L.C;
  a.smem_elems = (int)(L.smem_bytes / sizeof(S));
  a.tabs = P->d_tabs;
  a.piv = static_cast<const PV*>(P->d_piv);
  a.out = P->d_out;
  a.gstate = L.gstate ? static_cast<S*>(P->d_gstate) + L.gstate_off : nullptr;
  a.gstate_per_cta = L.gstate_per_cta;
  a.err = P->d_err;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(L.grid);
  cfg.blockDim = dim3(L.NT);
  cfg.dynamicSmemBytes = L.smem_bytes;
  cfg.stream = s;
  cudaLaunchAttribute attr;
  if (L.C > 1) {
    attr.id = cudaLaunchAttributeClusterDimension;
    attr.val.clusterDim.x = L.C;
    attr.val.clusterDim.y = 1;
    attr.val.clusterDim.z = 1;
    cfg.attrs = &attr;
    cfg.numAttrs = 1;
  }
  return cudaLaunchKernelEx(&cfg, rollback_fn<S, PV>(L.kind, L.NT, L.KX, L.gstate, L.full), a);
}

// Enqueue one run of a plan.  `ev` (optional) receives a start/stop event
// pair around each rollback launch.
cudaError_t plan_enqueue(lvc_plan* P, cudaStream_t s, cudaEvent_t* ev) {
  cudaError_t e = cudaMemsetAsync(P->d_err, 0, sizeof(int), s);
  if (e != cudaSuccess) return e;
  if (P->ncal == 0) return cudaSuccess;
  lvc_setup_kernel<<<P->ncal, 256, 0, s>>>(P->d_calibs, P->d_tabs);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if (P->row_start.back() > 0) {
    if (P->precision == LVC_F64)
      lvc_pivot_kernel<double><<<P->pivot_grid, 128, 0, s>>>(P->d_calibs, P->d_rowstart, P->ncal,
                                                              P->d_tabs, (double*)P->d_piv);
    else
      lvc_pivot_kernel<float><<<P->pivot_grid, 128, 0, s>>>(P->d_calibs, P->d_rowstart, P->ncal,
                                                             P->d_tabs, (float*)P->d_piv);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  for (size_t i = 0; i < P->launches.size(); i++) {
    const Launch& L = P->launches[i];
    if (L.n_items == 0) continue;
    if (ev && (e = cudaEventRecord(ev[2 * i], s)) != cudaSuccess) return e;
    e = P->precision == LVC_F64 ? launch_rollback<double, double>(P, L, s)
                                : launch_rollback<float, float>(P, L, s);
    if (e != cudaSuccess) return e;
    if (ev && (e = cudaEventRecord(ev[2 * i + 1], s)) != cudaSuccess) return e;
  }
  return cudaSuccess;
}

void plan_release(lvc_plan* P) {
  if (!P) return;
  if (P->exec) cudaGraphExecDestroy(P->exec);
  if (P->graph) cudaGraphDestroy(P->graph);
  cudaFree(P->d_calibs);
  cudaFree(P->d_tabs);
  cudaFree(P->d_piv);
  cudaFree(P->d_out);
  cudaFree(P->d_rowstart);
  cudaFree(P->d_items);
  cudaFree(P->d_gstate);
  cudaFree(P->d_err);
  delete P;
}

// Fills the per-calibration scalars (everything that depends on the inputs
// but not on the sizes).
void fill_scalars(CalibDev& d, const lvc_calibration& c) {
  d.s0 = c.s0;
  d.t = c.t;
  d.alpha = c.alpha;
  d.nu = c.nu;
  d.beta = c.beta;
  int xi = 0;
  spot_index(c.s0, c.alpha, c.t, c.numX, &xi);
  d.xindex = xi;
  d.yindex = c.numY / 2;
}

template <typename S, typename PV>
int plan_build(futhark_context* ctx, const lvc_calibration* cs, int n, lvc_plan* P) {
  P->ncal = n;
  P->params.assign(cs, cs + n);
  P->calibs.resize(n);
  P->row_start.assign(n + 1, 0);
  std::map<std::tuple<int, int, int, int, bool, bool>, std::vector<std::pair<int64_t, Item>>> classes;
  std::map<std::tuple<int, int, int, int, bool, bool>, Config> class_cfg;
  int64_t tab_off = 0, piv_off = 0, out_off = 0;
  for (int i = 0; i < n; i++) {
    const lvc_calibration& c = cs[i];
    if (int rc = validate(ctx, c, i)) return rc;
    const Config cf = choose_config<S>(c.numX, c.numY, ctx->max_smem);
    CalibDev& d = P->calibs[i];
    d.numX = c.numX;
    d.numY = c.numY;
    d.numT = c.numT;
    d.Xp = std::max(8, pow2ceil(c.numX));
    d.outer = c.outer;
    d.C = cf.C;
    d.kind = cf.kind;
    d.Ycs = cf.Ycs;
    d.pad0 = d.pad1 = 0;
    fill_scalars(d, c);
    d.tab = tab_off;
    tab_off += al2(tab_layout(c.numX, c.numY, c.numT, d.Xp, d.kind).total);
    d.piv = piv_off;
    piv_off += (piv_elems(c.numX, c.numY, c.numT, d.Xp, d.kind) + 3) & ~int64_t(3);
    d.out = out_off;
    out_off += c.outer;
    P->row_start[i + 1] = P->row_start[i] + (int64_t)(c.numT > 1 ? c.numT - 1 : 0) * c.numY;
    const auto key = std::make_tuple(cf.kind, cf.NT, cf.KX, cf.C, cf.gstate, cf.full);
    auto& cls = classes[key];
    auto it = class_cfg.find(key);
    if (it == class_cfg.end()) {
      class_cfg[key] = cf;
    } else {
      it->second.smem_bytes = std::max(it->second.smem_bytes, cf.smem_bytes);
      it->second.grid_elems = std::max(it->second.grid_elems, cf.grid_elems);
    }
    const int64_t cost = (int64_t)(c.numT > 1 ? c.numT - 1 : 0) * c.numX * c.numY;
    for (int s = 0; s < c.outer; s++) cls.push_back({cost, Item{i, s}});
  }
  P->tab_elems = tab_off;
  P->piv_elems = piv_off;
  P->nprices = out_off;
  // launch classes, largest work first inside each
  int64_t gstate_off = 0;
  for (auto& kv : classes) {
    auto& v = kv.second;
    std::stable_sort(v.begin(), v.end(),
                     [](const std::pair<int64_t, Item>& a, const std::pair<int64_t, Item>& b) {
                       return a.first > b.first;
                     });
    const Config& cf = class_cfg[kv.first];
    Launch L;
    L.kind = cf.kind;
    L.full = cf.full;
    L.NT = cf.NT;
    L.KX = cf.KX;
    L.C = cf.C;
    L.gstate = cf.gstate;
    L.item_off = (int)P->items.size();
    L.n_items = (int)v.size();
    L.smem_bytes = cf.smem_bytes;
    L.gstate_per_cta = cf.gstate ? cf.grid_elems : 0;
    for (auto& e : v) P->items.push_back(e.second);
    if (L.n_items > 0) {
      if (int rc = prepare_launch<S, PV>(ctx, L)) return rc;
    } else {
      L.grid = 0;
    }
    L.gstate_off = gstate_off;
    if (L.gstate) gstate_off += (int64_t)L.grid * L.gstate_per_cta;
    P->launches.push_back(L);
  }
  P->gstate_elems = gstate_off;
  const int64_t rows = P->row_start[n];
  P->pivot_grid = (int)std::max<int64_t>(1, std::min<int64_t>((rows + 127) / 128, 64LL * ctx->num_sms));

  // device buffers
  LVC_CUDA(ctx, cudaMalloc(&P->d_calibs, sizeof(CalibDev) * std::max(1, n)));
  LVC_CUDA(ctx, cudaMalloc(&P->d_tabs, sizeof(double) * std::max<int64_t>(2, P->tab_elems)));
  LVC_CUDA(ctx, cudaMalloc(&P->d_piv, sizeof(PV) * std::max<int64_t>(4, P->piv_elems)));
  LVC_CUDA(ctx, cudaMalloc(&P->d_out, sizeof(double) * std::max<int64_t>(1, P->nprices)));
  LVC_CUDA(ctx, cudaMalloc(&P->d_rowstart, sizeof(int64_t) * (n + 1)));
  LVC_CUDA(ctx, cudaMalloc(&P->d_items, sizeof(Item) * std::max<size_t>(1, P->items.size())));
  if (P->gstate_elems > 0) LVC_CUDA(ctx, cudaMalloc(&P->d_gstate, sizeof(S) * P->gstate_elems));
  LVC_CUDA(ctx, cudaMalloc(&P->d_err, sizeof(int)));
  if (n > 0)
    LVC_CUDA(ctx, cudaMemcpyAsync(P->d_calibs, P->calibs.data(), sizeof(CalibDev) * n,
                                  cudaMemcpyHostToDevice, ctx->stream));
  LVC_CUDA(ctx, cudaMemcpyAsync(P->d_rowstart, P->row_start.data(), sizeof(int64_t) * (n + 1),
                                cudaMemcpyHostToDevice, ctx->stream));
  if (!P->items.empty())
    LVC_CUDA(ctx, cudaMemcpyAsync(P->d_items, P->items.data(), sizeof(Item) * P->items.size(),
                                  cudaMemcpyHostToDevice, ctx->stream));
  LVC_CUDA(ctx, cudaMemsetAsync(P->d_out, 0, sizeof(double) * std::max<int64_t>(1, P->nprices),
                                ctx->stream));
  LVC_CUDA(ctx, cudaStreamSynchronize(ctx->stream));

  // capture one run into a graph
  LVC_CUDA(ctx, cudaStreamBeginCapture(ctx->capture, cudaStreamCaptureModeThreadLocal));
  cudaError_t e = plan_enqueue(P, ctx->capture, nullptr);
  cudaGraph_t g = nullptr;
  cudaError_t e2 = cudaStreamEndCapture(ctx->capture, &g);
  if (e != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return cuda_fail(ctx, e, "plan capture");
  }
  if (e2 != cudaSuccess) return cuda_fail(ctx, e2, "cudaStreamEndCapture");
  P->graph = g;
  LVC_CUDA(ctx, cudaGraphInstantiate(&P->exec, g, 0));
  return 0;
}

int plan_new_locked(futhark_context* ctx, const lvc_calibration* cs, int n, int precision,
                    lvc_plan** out) {
  if (!ctx->ok) return set_error(ctx, FUTHARK_PROGRAM_ERROR, "context has no usable CUDA device");
  if (n < 0 || (n > 0 && !cs)) return set_error(ctx, FUTHARK_PROGRAM_ERROR, "bad calibration list");
  if (precision != LVC_F64 && precision != LVC_F32_STATE)
    return set_error(ctx, FUTHARK_PROGRAM_ERROR, "unknown precision");
  LVC_CUDA(ctx, cudaSetDevice(ctx->device));
  lvc_plan* P = new lvc_plan();
  P->precision = precision;
  const int rc = precision == LVC_F64 ? plan_build<double, double>(ctx, cs, n, P)
                                      : plan_build<float, float>(ctx, cs, n, P);
  if (rc) {
    plan_release(P);
    return rc;
  }
  *out = P;
  return 0;
}

int check_device_error(futhark_context* ctx, lvc_plan* P) {
  int h = 0;
  LVC_CUDA(ctx, cudaMemcpyAsync(&h, P->d_err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  LVC_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (h) return set_error(ctx, FUTHARK_PROGRAM_ERROR, "rollback kernel rejected a work item");
  return 0;
}

int set_params_locked(futhark_context* ctx, lvc_plan* P, const lvc_calibration* cs, int n) {
  if (n != P->ncal) return set_error(ctx, FUTHARK_PROGRAM_ERROR, "calibration count changed");
  for (int i = 0; i < n; i++) {
    const lvc_calibration& a = P->params[i];
    const lvc_calibration& b = cs[i];
    if (a.outer != b.outer || a.numX != b.numX || a.numY != b.numY || a.numT != b.numT)
      return set_error(ctx, FUTHARK_PROGRAM_ERROR, "calibration sizes changed");
    if (int rc = validate(ctx, b, i)) return rc;
    fill_scalars(P->calibs[i], b);
    P->params[i] = b;
  }
  if (n > 0)
    LVC_CUDA(ctx, cudaMemcpyAsync(P->d_calibs, P->calibs.data(), sizeof(CalibDev) * n,
                                  cudaMemcpyHostToDevice, ctx->stream));
  return 0;
}

// The entry points run a one-calibration plan, kept while sizes repeat.
int entry_run(futhark_context* ctx, const lvc_calibration& c) {
  if (int rc = validate(ctx, c, 0)) return rc;
  lvc_plan* P = ctx->entry_plan;
  if (P) {
    const lvc_calibration& o = P->params[0];
    if (o.outer != c.outer || o.numX != c.numX || o.numY != c.numY || o.numT != c.numT) {
      LVC_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
      plan_release(P);
      P = ctx->entry_plan = nullptr;
    }
  }
  if (!P) {
    if (int rc = plan_new_locked(ctx, &c, 1, LVC_F64, &P)) return rc;
    ctx->entry_plan = P;
  } else if (int rc = set_params_locked(ctx, P, &c, 1)) {
    return rc;
  }
  LVC_CUDA(ctx, cudaGraphLaunch(P->exec, ctx->stream));
  return 0;
}

}  // namespace

extern "C" {

struct futhark_context_config* futhark_context_config_new(void) {
  return new (std::nothrow) futhark_context_config();
}
void futhark_context_config_free(struct futhark_context_config* cfg) { delete cfg; }
void futhark_context_config_set_device(struct futhark_context_config* cfg, const char* s) {
  if (!cfg || !s) return;
  if (s[0] == '#') {
    cfg->device = atoi(s + 1);
    cfg->device_name.clear();
  } else {
    cfg->device_name = s;
  }
}
void futhark_context_config_set_debugging(struct futhark_context_config* cfg, int flag) {
  if (cfg) cfg->debugging = flag;
}
void futhark_context_config_set_profiling(struct futhark_context_config* cfg, int flag) {
  if (cfg) cfg->profiling = flag;
}
void futhark_context_config_set_logging(struct futhark_context_config* cfg, int flag) {
  if (cfg) cfg->logging = flag;
}
void futhark_context_config_set_cache_file(struct futhark_context_config* cfg, const char* f) {
  (void)cfg;
  (void)f;
}

struct futhark_context* futhark_context_new(struct futhark_context_config* cfg) {
  futhark_context* ctx = new (std::nothrow) futhark_context();
  if (!ctx) return nullptr;
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) {
    ctx->error = std::string("no CUDA device: ") + cudaGetErrorString(e);
    return ctx;
  }
  int dev = cfg ? cfg->device : 0;
  if (cfg && !cfg->device_name.empty()) {
    dev = -1;
    for (int d = 0; d < ndev; d++) {
      cudaDeviceProp p;
      if (cudaGetDeviceProperties(&p, d) == cudaSuccess && strstr(p.name, cfg->device_name.c_str())) {
        dev = d;
        break;
      }
    }
    if (dev < 0) {
      ctx->error = "no CUDA device whose name contains \"" + cfg->device_name + "\"";
      return ctx;
    }
  }
  if (dev < 0 || dev >= ndev) {
    ctx->error = "CUDA device index out of range";
    return ctx;
  }
  cudaDeviceProp prop;
  if ((e = cudaSetDevice(dev)) != cudaSuccess || (e = cudaGetDeviceProperties(&prop, dev)) != cudaSuccess) {
    ctx->error = std::string("cannot use CUDA device: ") + cudaGetErrorString(e);
    return ctx;
  }
  if (prop.major < 10) {
    ctx->error = std::string("device ") + prop.name + " is not sm_100 (Blackwell); this build targets sm_100a";
    return ctx;
  }
  ctx->device = dev;
  ctx->num_sms = prop.multiProcessorCount;
  ctx->max_smem = (int)prop.sharedMemPerBlockOptin;
  if ((e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking)) != cudaSuccess ||
      (e = cudaStreamCreateWithFlags(&ctx->capture, cudaStreamNonBlocking)) != cudaSuccess) {
    ctx->error = std::string("cannot create stream: ") + cudaGetErrorString(e);
    return ctx;
  }
  ctx->ok = true;
  return ctx;
}

void futhark_context_free(struct futhark_context* ctx) {
  if (!ctx) return;
  if (ctx->ok) {
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    plan_release(ctx->entry_plan);
    cudaStreamDestroy(ctx->stream);
    cudaStreamDestroy(ctx->capture);
  }
  delete ctx;
}

int futhark_context_sync(struct futhark_context* ctx) {
  std::lock_guard<std::mutex> g(ctx->mu);
  if (!ctx->ok) return set_error(ctx, FUTHARK_PROGRAM_ERROR, "context has no usable CUDA device");
  LVC_CUDA(ctx, cudaSetDevice(ctx->device));
  LVC_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return 0;
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
  LVC_CUDA(ctx, cudaSetDevice(ctx->device));
  LVC_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  plan_release(ctx->entry_plan);
  ctx->entry_plan = nullptr;
  return 0;
}

#define LVC_ARRAY_FUNCS(T, NAME)                                                                 \
  struct futhark_##NAME##_1d* futhark_new_##NAME##_1d(struct futhark_context* ctx, const T* data, \
                                                      int64_t dim0) {                            \
    std::lock_guard<std::mutex> g(ctx->mu);                                                      \
    if (!ctx->ok || dim0 < 0) {                                                                  \
      ctx->error = "cannot create array";                                                       \
      return nullptr;                                                                            \
    }                                                                                            \
    cudaSetDevice(ctx->device);                                                                  \
    auto* a = new (std::nothrow) futhark_##NAME##_1d();                                          \
    if (!a) return nullptr;                                                                      \
    a->shape[0] = dim0;                                                                          \
    a->bytes = sizeof(T) * (size_t)std::max<int64_t>(1, dim0);                                   \
    if (cudaMalloc(&a->data, a->bytes) != cudaSuccess) {                                         \
      ctx->error = "out of device memory";                                                       \
      delete a;                                                                                  \
      return nullptr;                                                                            \
    }                                                                                            \
    if (dim0 > 0 && data &&                                                                      \
        cudaMemcpyAsync(a->data, data, sizeof(T) * dim0, cudaMemcpyHostToDevice, ctx->stream) != \
            cudaSuccess) {                                                                       \
      cudaFree(a->data);                                                                         \
      delete a;                                                                                  \
      ctx->error = "host to device copy failed";                                                 \
      return nullptr;                                                                            \
    }                                                                                            \
    cudaStreamSynchronize(ctx->stream);                                                          \
    return a;                                                                                    \
  }                                                                                              \
  int futhark_free_##NAME##_1d(struct futhark_context* ctx, struct futhark_##NAME##_1d* arr) {   \
    if (!arr) return 0;                                                                          \
    std::lock_guard<std::mutex> g(ctx->mu);                                                      \
    cudaSetDevice(ctx->device);                                                                  \
    cudaStreamSynchronize(ctx->stream);                                                          \
    cudaFree(arr->data);                                                                         \
    delete arr;                                                                                  \
    return 0;                                                                                    \
  }                                                                                              \
  int futhark_values_##NAME##_1d(struct futhark_context* ctx, struct futhark_##NAME##_1d* arr,   \
                                 T* data) {                                                      \
    std::lock_guard<std::mutex> g(ctx->mu);                                                      \
    if (!arr) return set_error(ctx, FUTHARK_PROGRAM_ERROR, "null array");                        \
    LVC_CUDA(ctx, cudaSetDevice(ctx->device));                                                   \
    if (arr->shape[0] > 0)                                                                       \
      LVC_CUDA(ctx, cudaMemcpyAsync(data, arr->data, sizeof(T) * arr->shape[0],                 \
                                    cudaMemcpyDeviceToHost, ctx->stream));                       \
    LVC_CUDA(ctx, cudaStreamSynchronize(ctx->stream));                                           \
    return 0;                                                                                    \
  }                                                                                              \
  const int64_t* futhark_shape_##NAME##_1d(struct futhark_context* ctx,                          \
                                           struct futhark_##NAME##_1d* arr) {                    \
    (void)ctx;                                                                                   \
    return arr ? arr->shape : nullptr;                                                           \
  }

LVC_ARRAY_FUNCS(float, f32)
LVC_ARRAY_FUNCS(double, f64)

int futhark_entry_main_f64(struct futhark_context* ctx, struct futhark_f64_1d** out0,
                           const int32_t outer, const int32_t numX, const int32_t numY,
                           const int32_t numT, const double s0, const double t, const double alpha,
                           const double nu, const double beta) {
  std::lock_guard<std::mutex> g(ctx->mu);
  if (!ctx->ok) return set_error(ctx, FUTHARK_PROGRAM_ERROR, "context has no usable CUDA device");
  LVC_CUDA(ctx, cudaSetDevice(ctx->device));
  const lvc_calibration c{outer, numX, numY, numT, s0, t, alpha, nu, beta};
  if (int rc = entry_run(ctx, c)) return rc;
  auto* a = new (std::nothrow) futhark_f64_1d();
  if (!a) return set_error(ctx, FUTHARK_OUT_OF_MEMORY, "host allocation failed");
  a->shape[0] = outer;
  a->bytes = sizeof(double) * (size_t)std::max(1, outer);
  cudaError_t e = cudaMalloc(&a->data, a->bytes);
  if (e != cudaSuccess) {
    delete a;
    return cuda_fail(ctx, e, "cudaMalloc");
  }
  if (outer > 0 && (e = cudaMemcpyAsync(a->data, ctx->entry_plan->d_out, sizeof(double) * outer,
                                        cudaMemcpyDeviceToDevice, ctx->stream)) != cudaSuccess) {
    cudaFree(a->data);
    delete a;
    return cuda_fail(ctx, e, "cudaMemcpyAsync");
  }
  if (int rc = check_device_error(ctx, ctx->entry_plan)) {
    cudaFree(a->data);
    delete a;
    return rc;
  }
  *out0 = a;
  return 0;
}

int futhark_entry_main(struct futhark_context* ctx, struct futhark_f32_1d** out0,
                       const int32_t outer, const int32_t numX, const int32_t numY,
                       const int32_t numT, const float s0, const float t, const float alpha,
                       const float nu, const float beta) {
  std::lock_guard<std::mutex> g(ctx->mu);
  if (!ctx->ok) return set_error(ctx, FUTHARK_PROGRAM_ERROR, "context has no usable CUDA device");
  LVC_CUDA(ctx, cudaSetDevice(ctx->device));
  const lvc_calibration c{outer, numX, numY, numT, s0, t, alpha, nu, beta};
  if (int rc = entry_run(ctx, c)) return rc;
  auto* a = new (std::nothrow) futhark_f32_1d();
  if (!a) return set_error(ctx, FUTHARK_OUT_OF_MEMORY, "host allocation failed");
  a->shape[0] = outer;
  a->bytes = sizeof(float) * (size_t)std::max(1, outer);
  cudaError_t e = cudaMalloc(&a->data, a->bytes);
  if (e != cudaSuccess) {
    delete a;
    return cuda_fail(ctx, e, "cudaMalloc");
  }
  if (outer > 0) {
    lvc_to_f32_kernel<<<(outer + 255) / 256, 256, 0, ctx->stream>>>(ctx->entry_plan->d_out, a->data,
                                                                     outer);
    if ((e = cudaGetLastError()) != cudaSuccess) {
      cudaFree(a->data);
      delete a;
      return cuda_fail(ctx, e, "lvc_to_f32_kernel");
    }
  }
  if (int rc = check_device_error(ctx, ctx->entry_plan)) {
    cudaFree(a->data);
    delete a;
    return rc;
  }
  *out0 = a;
  return 0;
}

int lvc_plan_new(struct futhark_context* ctx, const struct lvc_calibration* calibs, int32_t n,
                 int32_t precision, struct lvc_plan** plan) {
  std::lock_guard<std::mutex> g(ctx->mu);
  return plan_new_locked(ctx, calibs, n, precision, plan);
}

int lvc_plan_free(struct futhark_context* ctx, struct lvc_plan* plan) {
  std::lock_guard<std::mutex> g(ctx->mu);
  if (ctx->ok) {
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
  }
  plan_release(plan);
  return 0;
}

int64_t lvc_plan_num_prices(const struct lvc_plan* plan) { return plan ? plan->nprices : 0; }

int lvc_plan_set_params(struct futhark_context* ctx, struct lvc_plan* plan,
                        const struct lvc_calibration* calibs, int32_t n) {
  std::lock_guard<std::mutex> g(ctx->mu);
  LVC_CUDA(ctx, cudaSetDevice(ctx->device));
  return set_params_locked(ctx, plan, calibs, n);
}

int lvc_plan_run(struct futhark_context* ctx, struct lvc_plan* plan) {
  std::lock_guard<std::mutex> g(ctx->mu);
  LVC_CUDA(ctx, cudaSetDevice(ctx->device));
  LVC_CUDA(ctx, cudaGraphLaunch(plan->exec, ctx->stream));
  return 0;
}

int lvc_plan_copy_prices(struct futhark_context* ctx, struct lvc_plan* plan, double* prices) {
  std::lock_guard<std::mutex> g(ctx->mu);
  LVC_CUDA(ctx, cudaSetDevice(ctx->device));
  if (plan->nprices > 0)
    LVC_CUDA(ctx, cudaMemcpyAsync(prices, plan->d_out, sizeof(double) * plan->nprices,
                                  cudaMemcpyDeviceToHost, ctx->stream));
  return check_device_error(ctx, plan);
}

const double* lvc_plan_device_prices(const struct lvc_plan* plan) { return plan ? plan->d_out : nullptr; }

int32_t lvc_plan_num_launches(const struct lvc_plan* plan) {
  if (!plan || plan->ncal == 0) return 0;
  int32_t n = 1 + (plan->row_start.back() > 0 ? 1 : 0);
  for (const auto& L : plan->launches) n += L.n_items > 0 ? 1 : 0;
  return n;
}

int lvc_plan_time(struct futhark_context* ctx, struct lvc_plan* plan, int32_t iters,
                  double* ms_per_run) {
  std::lock_guard<std::mutex> g(ctx->mu);
  LVC_CUDA(ctx, cudaSetDevice(ctx->device));
  if (iters < 1) iters = 1;
  cudaEvent_t a, b;
  LVC_CUDA(ctx, cudaEventCreate(&a));
  LVC_CUDA(ctx, cudaEventCreate(&b));
  LVC_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  LVC_CUDA(ctx, cudaEventRecord(a, ctx->stream));
  for (int i = 0; i < iters; i++) LVC_CUDA(ctx, cudaGraphLaunch(plan->exec, ctx->stream));
  LVC_CUDA(ctx, cudaEventRecord(b, ctx->stream));
  LVC_CUDA(ctx, cudaEventSynchronize(b));
  float ms = 0.f;
  LVC_CUDA(ctx, cudaEventElapsedTime(&ms, a, b));
  *ms_per_run = ms / iters;
  // the rollback launches alone, with events between the kernels
  std::vector<cudaEvent_t> ev(2 * plan->launches.size());
  for (auto& x : ev) LVC_CUDA(ctx, cudaEventCreate(&x));
  double roll = 0.0;
  for (int i = 0; i < iters; i++) {
    cudaError_t e = plan_enqueue(plan, ctx->stream, ev.data());
    if (e != cudaSuccess) return cuda_fail(ctx, e, "plan_enqueue");
    LVC_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    for (size_t l = 0; l < plan->launches.size(); l++) {
      if (plan->launches[l].n_items == 0) continue;
      float t = 0.f;
      LVC_CUDA(ctx, cudaEventElapsedTime(&t, ev[2 * l], ev[2 * l + 1]));
      roll += t;
    }
  }
  plan->rollback_ms = roll / iters;
  for (auto& x : ev) cudaEventDestroy(x);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return check_device_error(ctx, plan);
}

double lvc_plan_rollback_ms(const struct lvc_plan* plan) { return plan ? plan->rollback_ms : 0.0; }

int lvc_batch(struct futhark_context* ctx, const struct lvc_calibration* calibs, int32_t n,
              int32_t precision, double* prices) {
  lvc_plan* P = nullptr;
  if (int rc = lvc_plan_new(ctx, calibs, n, precision, &P)) return rc;
  int rc = lvc_plan_run(ctx, P);
  if (!rc) rc = lvc_plan_copy_prices(ctx, P, prices);
  lvc_plan_free(ctx, P);
  return rc;
}

void* lvc_context_stream(struct futhark_context* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

int lvc_probe_peaks(struct futhark_context* ctx, double* fp64_tflops, double* smem_gbs) {
  std::lock_guard<std::mutex> g(ctx->mu);
  if (!ctx->ok) return set_error(ctx, FUTHARK_PROGRAM_ERROR, "context has no usable CUDA device");
  LVC_CUDA(ctx, cudaSetDevice(ctx->device));
  void* scratch = nullptr;
  LVC_CUDA(ctx, cudaMalloc(&scratch, 1 << 20));
  cudaEvent_t a, b;
  LVC_CUDA(ctx, cudaEventCreate(&a));
  LVC_CUDA(ctx, cudaEventCreate(&b));
  const int dgrid = ctx->num_sms * 8, diters = 20000;
  const int sgrid = ctx->num_sms * 4, siters = 20000;
  float best_d = 1e30f, best_s = 1e30f;
  for (int rep = 0; rep < 4; rep++) {
    float ms = 0.f;
    LVC_CUDA(ctx, cudaEventRecord(a, ctx->stream));
    lvc_probe_dfma_kernel<<<dgrid, 256, 0, ctx->stream>>>((double*)scratch, diters, 0.9999999, 1e-7);
    LVC_CUDA(ctx, cudaGetLastError());
    LVC_CUDA(ctx, cudaEventRecord(b, ctx->stream));
    LVC_CUDA(ctx, cudaEventSynchronize(b));
    LVC_CUDA(ctx, cudaEventElapsedTime(&ms, a, b));
    if (rep > 0) best_d = std::min(best_d, ms);
    LVC_CUDA(ctx, cudaEventRecord(a, ctx->stream));
    lvc_probe_smem_kernel<<<sgrid, 512, 0, ctx->stream>>>((unsigned long long*)scratch, siters);
    LVC_CUDA(ctx, cudaGetLastError());
    LVC_CUDA(ctx, cudaEventRecord(b, ctx->stream));
    LVC_CUDA(ctx, cudaEventSynchronize(b));
    LVC_CUDA(ctx, cudaEventElapsedTime(&ms, a, b));
    if (rep > 0) best_s = std::min(best_s, ms);
  }
  const double flops = 2.0 * kProbeChains * (double)diters * 256.0 * dgrid;
  const double bytes = 16.0 * 4.0 * (double)siters * 512.0 * sgrid;
  *fp64_tflops = flops / (best_d * 1e-3) / 1e12;
  *smem_gbs = bytes / (best_s * 1e-3) / 1e9;
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(scratch);
  return 0;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Entry point without device allocation.
//
// Some callers cannot call cudaMalloc at the moment they need a price: a
// serving loop that must never trigger the implicit device synchronisation of
// cudaMalloc/cudaFree, code running under a caching allocator or a memory
// budget that owns every byte of the device, or a host that has already handed
// the rest of HBM to other work.  For them lvc_entry_main_f64_noalloc runs
// the same setup, pivot and rollback kernels as futhark_entry_main_f64, with
// every scratch buffer (calibration record, work list, operator tables, pivot
// rows, error flag) carved from one fixed static device array instead of
// device allocations.  The array exists once per device that loads this
// library and is held until the process exits.
// ---------------------------------------------------------------------------
namespace {

constexpr size_t kNoAllocScratchBytes = (size_t)LVC_NOALLOC_SCRATCH_BYTES;
static __device__ __align__(256) unsigned char lvc_noalloc_scratch[kNoAllocScratchBytes];

// Device address of lvc_noalloc_scratch, looked up once per device.  In host
// code the symbol is only a host-side stand-in; kernels must be given this
// address.
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
void* g_noalloc_addr[kMaxDevices] = {};

int noalloc_scratch(futhark_context* ctx, unsigned char** out) {
  if (ctx->device < 0 || ctx->device >= kMaxDevices)
    return set_error(ctx, FUTHARK_PROGRAM_ERROR, "device ordinal out of range for the static scratch");
  std::lock_guard<std::mutex> g(g_noalloc_mu);
  if (!g_noalloc_addr[ctx->device]) {
    void* p = nullptr;  // the current device is ctx->device (set by the caller)
    cudaError_t e = cudaGetSymbolAddress(&p, lvc_noalloc_scratch);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaGetSymbolAddress(lvc_noalloc_scratch)");
    if (!p) return set_error(ctx, FUTHARK_PROGRAM_ERROR, "static scratch has no device address");
    g_noalloc_addr[ctx->device] = p;
  }
  *out = static_cast<unsigned char*>(g_noalloc_addr[ctx->device]);
  return 0;
}

__global__ void lvc_noalloc_items_kernel(Item* items, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    items[i] = Item{0, i};
}

size_t up256(size_t n) { return (n + 255) & ~size_t(255); }

}  // namespace

extern "C" int lvc_entry_main_f64_noalloc(struct futhark_context* ctx, double* prices,
                                          const int32_t outer, const int32_t numX,
                                          const int32_t numY, const int32_t numT, const double s0,
                                          const double t, const double alpha, const double nu,
                                          const double beta) {
  std::lock_guard<std::mutex> g(ctx->mu);
  if (!ctx->ok) return set_error(ctx, FUTHARK_PROGRAM_ERROR, "context has no usable CUDA device");
  LVC_CUDA(ctx, cudaSetDevice(ctx->device));
  const lvc_calibration c{outer, numX, numY, numT, s0, t, alpha, nu, beta};
  if (int rc = validate(ctx, c, 0)) return rc;
  if (outer > 0 && !prices) return set_error(ctx, FUTHARK_PROGRAM_ERROR, "null price buffer");
  unsigned char* base = nullptr;
  if (int rc = noalloc_scratch(ctx, &base)) return rc;

  const Config cf = choose_config<double>(numX, numY, ctx->max_smem);
  if (cf.gstate)
    return set_error(ctx, FUTHARK_PROGRAM_ERROR,
                     "lvc_entry_main_f64_noalloc: this grid does not fit on chip; its HBM state "
                     "needs the allocating entry point futhark_entry_main_f64");
  CalibDev d;
  memset(&d, 0, sizeof d);
  d.numX = numX;
  d.numY = numY;
  d.numT = numT;
  d.Xp = std::max(8, pow2ceil(numX));
  d.outer = outer;
  d.C = cf.C;
  d.kind = cf.kind;
  d.Ycs = cf.Ycs;
  fill_scalars(d, c);
  d.tab = 0;
  d.piv = 0;
  d.out = 0;
  const int64_t tab_elems = al2(tab_layout(numX, numY, numT, d.Xp, d.kind).total);
  const int64_t piv_n = (piv_elems(numX, numY, numT, d.Xp, d.kind) + 3) & ~int64_t(3);
  // scratch carve-up
  const size_t o_calib = 0;
  const size_t o_err = up256(o_calib + sizeof(CalibDev));
  const size_t o_rows = up256(o_err + sizeof(int));
  const size_t o_items = up256(o_rows + 2 * sizeof(int64_t));
  const size_t o_tabs = up256(o_items + sizeof(Item) * (size_t)std::max(1, outer));
  const size_t o_piv = up256(o_tabs + sizeof(double) * (size_t)tab_elems);
  const size_t need = o_piv + sizeof(double) * (size_t)piv_n;
  if (need > kNoAllocScratchBytes) {
    char buf[256];
    snprintf(buf, sizeof buf,
             "lvc_entry_main_f64_noalloc: this calibration needs %zu bytes of scratch, more than "
             "the static %zu bytes; use futhark_entry_main_f64",
             need, kNoAllocScratchBytes);
    return set_error(ctx, FUTHARK_PROGRAM_ERROR, buf);
  }
  CalibDev* d_calib = reinterpret_cast<CalibDev*>(base + o_calib);
  int* d_err = reinterpret_cast<int*>(base + o_err);
  int64_t* d_rows = reinterpret_cast<int64_t*>(base + o_rows);
  Item* d_items = reinterpret_cast<Item*>(base + o_items);
  double* d_tabs = reinterpret_cast<double*>(base + o_tabs);
  double* d_piv = reinterpret_cast<double*>(base + o_piv);
  const int64_t rows[2] = {0, (int64_t)(numT > 1 ? numT - 1 : 0) * numY};
  cudaStream_t s = ctx->stream;

  // the array keeps the previous call's contents: reset what must start at zero
  LVC_CUDA(ctx, cudaMemsetAsync(d_err, 0, sizeof(int), s));
  LVC_CUDA(ctx, cudaMemcpyAsync(d_calib, &d, sizeof d, cudaMemcpyHostToDevice, s));
  LVC_CUDA(ctx, cudaMemcpyAsync(d_rows, rows, sizeof rows, cudaMemcpyHostToDevice, s));
  if (outer > 0) {
    lvc_noalloc_items_kernel<<<(outer + 255) / 256, 256, 0, s>>>(d_items, outer);
    LVC_CUDA(ctx, cudaGetLastError());
  }
  lvc_setup_kernel<<<1, 256, 0, s>>>(d_calib, d_tabs);
  LVC_CUDA(ctx, cudaGetLastError());
  if (rows[1] > 0) {
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((rows[1] + 127) / 128, 64LL * ctx->num_sms));
    lvc_pivot_kernel<double><<<grid, 128, 0, s>>>(d_calib, d_rows, 1, d_tabs, d_piv);
    LVC_CUDA(ctx, cudaGetLastError());
  }
  if (outer > 0) {
    Launch L;
    L.kind = cf.kind;
    L.full = cf.full;
    L.NT = cf.NT;
    L.KX = cf.KX;
    L.C = cf.C;
    L.gstate = false;
    L.item_off = 0;
    L.n_items = outer;
    L.smem_bytes = cf.smem_bytes;
    L.gstate_per_cta = 0;
    L.gstate_off = 0;
    if (int rc = prepare_launch<double, double>(ctx, L)) return rc;
    RollbackArgs<double, double> a;
    a.calibs = d_calib;
    a.items = d_items;
    a.n_items = outer;
    a.C = L.C;
    a.smem_elems = (int)(L.smem_bytes / sizeof(double));
    a.tabs = d_tabs;
    a.piv = d_piv;
    a.out = prices;
    a.gstate = nullptr;
    a.gstate_per_cta = 0;
    a.err = d_err;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(L.grid);
    cfg.blockDim = dim3(L.NT);
    cfg.dynamicSmemBytes = L.smem_bytes;
    cfg.stream = s;
    cudaLaunchAttribute attr;
    if (L.C > 1) {
      attr.id = cudaLaunchAttributeClusterDimension;
      attr.val.clusterDim.x = L.C;
      attr.val.clusterDim.y = 1;
      attr.val.clusterDim.z = 1;
      cfg.attrs = &attr;
      cfg.numAttrs = 1;
    }
    LVC_CUDA(ctx, cudaLaunchKernelEx(&cfg, rollback_fn<double, double>(L.kind, L.NT, L.KX, false, L.full), a));
  }
  int h = 0;
  LVC_CUDA(ctx, cudaMemcpyAsync(&h, d_err, sizeof(int), cudaMemcpyDeviceToHost, s));
  LVC_CUDA(ctx, cudaStreamSynchronize(s));
  if (h) return set_error(ctx, FUTHARK_PROGRAM_ERROR, "rollback kernel rejected a work item");
  return 0;
}
