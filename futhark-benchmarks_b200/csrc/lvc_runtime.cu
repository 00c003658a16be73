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
//   * one run = setup kernel + pivot kernel + one rollback launch per class,
//     the classes forked over several streams (largest class first) so their
//     tails overlap, captured once into a CUDA graph.
#include <cuda_runtime.h>
#include <cudaTypedefs.h>  // the driver's cuTensorMapEncodeTiled signature

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <deque>
#include <thread>
#include <unordered_map>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <set>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "LocVolCalib.h"
#include "lvc_kernels.cuh"
#include "lvc_line.cuh"
#include "lvc_pair.cuh"
#include "lvc_tridiag.cuh"
#include "tridiag.h"
#include "lvc_probe.cuh"

using namespace lvc;

// Tuning parameters, set by name as in Futhark's generated API
// (futhark_context_config_set_tuning_param) or on a live context.
//   lvc.streams  streams a batch plan forks its launch classes over (1..8)
//   lvc.grid     0: persistent grids sized to the resident CTAs, items taken
//                in strides; 1: one CTA (cluster) per strike instance, the
//                block scheduler handing out items in descending work order;
//                2: 0 for f64 plans, 1 for f32-state plans (the measured best
//                of each on the uneven calibration mix)
struct TuningParams {
  int streams = 4;
  int grid = 2;
};

int grid_mode(const TuningParams& t, int precision) {
  return t.grid == 2 ? (precision == LVC_F32_STATE ? 1 : 0) : t.grid;
}
const char* const kTuningNames[] = {"lvc.streams", "lvc.grid"};
const char* const kTuningClasses[] = {"streams", "grid"};
constexpr int kNumTuning = 2;
constexpr int kMaxNumX = 512;   // largest grid the kernels take
constexpr int kMaxNumY = 1024;
constexpr int kMaxAux = 8;

int set_tuning(TuningParams& t, const char* name, size_t v) {
  if (!name) return 1;
  if (!strcmp(name, "lvc.streams")) {
    if (v < 1 || v > (size_t)kMaxAux) return 1;
    t.streams = (int)v;
    return 0;
  }
  if (!strcmp(name, "lvc.grid")) {
    if (v > 2) return 1;
    t.grid = (int)v;
    return 0;
  }
  return 1;
}

struct futhark_context_config {
  int device = 0;
  std::string device_name;
  int debugging = 0, profiling = 0, logging = 0;
  TuningParams tuning;
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
struct futhark_f32_2d {
  float* data;
  int64_t shape[2];
  size_t bytes;
};

namespace {

// Pool of device memory.  Plans (batch, entry point, serving) take their
// buffers from a pool, so steady-state calls do not reach cudaMalloc/cudaFree
// (which synchronise the device; freeing a batch plan's 10 GB of pivot rows
// took most of a second).  Small requests are carved first-fit out of
// 256 MB chunks; a request of a chunk or more gets a block of its own, which
// is kept for later large requests (best fit) when released.  When the
// device has no room left, blocks that are entirely free are returned to
// CUDA (trim) and the allocation is retried.  With a budget, allocation fails
// instead of growing past it -- the serving runtime's HBM admission control.
struct DevicePool {
  std::mutex mu;
  size_t budget = 0;               // 0: unlimited
  size_t chunk = size_t(256) << 20;
  std::map<char*, size_t> blocks;  // start -> size of every block from cudaMalloc
  std::map<char*, size_t> large;   // blocks of a single large request (subset of blocks)
  std::map<char*, size_t> free_;   // start -> size, in chunk blocks
  std::map<char*, size_t> large_free;
  std::map<char*, size_t> used_;
  size_t reserved = 0, in_use = 0;

  ~DevicePool() {
    for (auto& b : blocks) cudaFree(b.first);
  }
  char* grow(size_t sz) {
    if (budget && reserved + sz > budget) return nullptr;
    char* p = nullptr;
    if (cudaMalloc(&p, sz) != cudaSuccess) {
      cudaGetLastError();
      if (!trim_locked()) return nullptr;
      if (budget && reserved + sz > budget) return nullptr;
      if (cudaMalloc(&p, sz) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
      }
    }
    blocks[p] = sz;
    reserved += sz;
    return p;
  }
  // Returns every entirely free block to CUDA; true if any was released.
  bool trim_locked() {
    bool any = false;
    for (auto it = large_free.begin(); it != large_free.end();) {
      cudaFree(it->first);
      reserved -= it->second;
      blocks.erase(it->first);
      large.erase(it->first);
      it = large_free.erase(it);
      any = true;
    }
    for (auto it = blocks.begin(); it != blocks.end();) {
      auto f = free_.find(it->first);
      if (!large.count(it->first) && f != free_.end() && f->second == it->second) {
        cudaFree(it->first);
        reserved -= it->second;
        free_.erase(f);
        it = blocks.erase(it);
        any = true;
      } else {
        ++it;
      }
    }
    return any;
  }
  void trim() {
    std::lock_guard<std::mutex> g(mu);
    trim_locked();
  }
  void insert_free(char* p, size_t sz) {
    auto nx = free_.lower_bound(p);
    if (nx != free_.end() && p + sz == nx->first) {
      sz += nx->second;
      nx = free_.erase(nx);
    }
    if (nx != free_.begin()) {
      auto pv = std::prev(nx);
      if (pv->first + pv->second == p) {
        pv->second += sz;
        return;
      }
    }
    free_[p] = sz;
  }
  void* alloc(size_t bytes) {
    bytes = (std::max<size_t>(bytes, 1) + 255) & ~size_t(255);
    std::lock_guard<std::mutex> g(mu);
    if (bytes >= chunk && !budget) {
      // best fit among the released large blocks, else a block of its own
      // (a budgeted pool carves everything out of its chunks)
      auto best = large_free.end();
      for (auto it = large_free.begin(); it != large_free.end(); ++it)
        if (it->second >= bytes && (best == large_free.end() || it->second < best->second)) best = it;
      char* p = nullptr;
      size_t sz = 0;
      if (best != large_free.end()) {
        p = best->first;
        sz = best->second;
        large_free.erase(best);
      } else {
        sz = (bytes + (size_t(2) << 20) - 1) & ~((size_t(2) << 20) - 1);
        if (!(p = grow(sz))) return nullptr;
        large[p] = sz;
      }
      used_[p] = sz;
      in_use += sz;
      return p;
    }
    for (int attempt = 0; attempt < 2; attempt++) {
      for (auto it = free_.begin(); it != free_.end(); ++it) {
        if (it->second >= bytes) {
          char* p = it->first;
          const size_t rem = it->second - bytes;
          free_.erase(it);
          if (rem) free_[p + bytes] = rem;
          used_[p] = bytes;
          in_use += bytes;
          return p;
        }
      }
      if (attempt == 0) {
        size_t sz = chunk;
        if (budget && reserved + sz > budget) sz = bytes;
        char* p = grow(sz);
        if (!p) return nullptr;
        insert_free(p, sz);
      }
    }
    return nullptr;
  }
  void release(void* vp) {
    if (!vp) return;
    std::lock_guard<std::mutex> g(mu);
    auto it = used_.find(static_cast<char*>(vp));
    if (it == used_.end()) return;
    const size_t sz = it->second;
    used_.erase(it);
    in_use -= sz;
    if (large.count(static_cast<char*>(vp)))
      large_free[static_cast<char*>(vp)] = sz;
    else
      insert_free(static_cast<char*>(vp), sz);
  }
};

// Kernel configuration of one calibration.
struct Config {
  int kind, NT, KX, C;
  bool gstate;
  bool full = false;
  bool pair = false;  // paired line kernel
  int upw = 2;        // paired kernel: units per warp
  int ld = 0;         // line family: row stride of the pivot rows and the on-chip grid
  int Ycs;
  size_t smem_bytes;
  int64_t grid_elems;
};

// A tuned grid class: the configuration chosen for (numX, numY, precision).
struct TunedShape {
  Config cf;
  bool tuned = false;
  double us_default = 0.0, us_best = 0.0;
};

struct Launch {
  int kind, NT, KX, C;
  bool gstate;
  bool full = false;
  bool pair = false;
  int upw = 2;
  int item_off, n_items, grid;
  size_t smem_bytes;
  int64_t gstate_per_cta;  // elements of the state type
  int64_t gstate_off;      // elements
  double sm_per_cta = 1.0; // SMs one CTA of this launch occupies at full residency
  int64_t work = 0;        // option-cell-steps of the launch's items
  double ms = 0.0;         // device time in the last lvc_plan_time (mean per run)
};

}  // namespace

struct lvc_plan {
  int precision = LVC_F64;
  int ncal = 0;
  int64_t nprices = 0;
  std::vector<lvc_calibration> params;
  std::vector<CalibDev> calibs;
  std::vector<Config> cfgs;  // the shape each calibration runs under
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
  DevicePool* pool = nullptr;  // where the buffers come from (null: cudaMalloc)
  bool use_graph = true;       // capture one run into a CUDA graph
  int max_sms = 0;             // cap on the SMs a launch may occupy (0: all, <0: one CTA per item)
  double sms = 0.0;            // SMs the widest launch occupies
  int n_streams = 1;           // streams the launch classes fork over
  uint64_t shapes_gen = 0;     // the context's tuning-table generation the plan was built under
  cudaStream_t aux[kMaxAux] = {};
  cudaEvent_t ev_fork = nullptr;
  cudaEvent_t ev_join[kMaxAux] = {};
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
  DevicePool* pool = nullptr;      // buffers of the entry points' plans
  TuningParams tuning;
  cudaStream_t aux[kMaxAux] = {};  // fork streams of the batch plans
  std::map<std::tuple<int, int, int>, TunedShape> shapes;  // (numX, numY, precision) -> tuned shape
  uint64_t shapes_gen = 0;  // bumped on every change of `shapes`
  // tridiagonal solves: the tensor maps of the last batch that took the
  // tensor-copy kernel, reused while its four inputs and shape repeat, and
  // the kernels whose shared-memory limit is already raised on this device
  const float* tri_map_src[4] = {};
  int64_t tri_map_rows = -1, tri_map_m = -1;
  CUtensorMap tri_maps[4];
  std::set<const void*> tri_smem_raised;
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
  if (c.numX > kMaxNumX || c.numY > kMaxNumY) {
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
RbFn<S, PV> rollback_fn(int kind, int NT, int KX, bool gs, bool full = false, bool pair = false,
                        int upw = 2) {
  if (kind == kKindLine && pair && upw == 1) {
    if (NT == 64) return lvc_line_pair_kernel<S, PV, 64, 1>;
    if (NT == 128) return lvc_line_pair_kernel<S, PV, 128, 1>;
    if (NT == 256) return lvc_line_pair_kernel<S, PV, 256, 1>;
    if (NT == 512) return lvc_line_pair_kernel<S, PV, 512, 1>;
    return nullptr;
  }
  if (kind == kKindLine && pair) {
    if (NT == 64) return lvc_line_pair_kernel<S, PV, 64, 2>;
    if (NT == 128) return lvc_line_pair_kernel<S, PV, 128, 2>;
    if (NT == 256) return lvc_line_pair_kernel<S, PV, 256, 2>;
    return nullptr;
  }
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


// Line family, full tiles: every line chunk, row group and CTA block
// complete; two units per warp, one unit per 512 cells.
template <typename S>
bool line_full_cfg(int X, int Y, int C, int max_smem, Config& cf) {
  if (X > 256 || X % 32 || Y % C || (Y / C) % 32) return false;
  const int Ycs = Y / C;
  const int units = X * Ycs / 512;
  if (units != 2 && units != 4 && units != 8 && units != 16) return false;  // NT = 16 * units instantiated
  const FullLayout F = full_layout<S>(X, Ycs, units);
  if (F.Ux != units || F.Uy != units || F.total > max_smem) return false;
  cf.kind = kKindLine;
  cf.full = true;
  cf.pair = false;
  cf.ld = line_ld(X);
  cf.NT = 16 * units;  // 32 lanes x units / 2 units per warp
  cf.KX = kLineK;
  cf.C = C;
  cf.gstate = false;
  cf.Ycs = Ycs;
  cf.smem_bytes = (size_t)F.total;
  cf.grid_elems = 0;
  return true;
}

// Paired line kernel on full tiles: upw = 2 (two X units and one 64-column
// Y unit per warp, numX % 64 == 0) or upw = 1 (one X unit and one 32-column
// Y unit per warp, twice the warps).
template <typename S>
bool line_pair_cfg(int X, int Y, int C, int max_smem, Config& cf, int upw = 2) {
  if (X > 256 || X % (32 * upw) || Y % C || (Y / C) % 32) return false;
  const int Ycs = Y / C;
  const int units = X * Ycs / 512;  // X units of 32 rows x 16 columns
  const int NW = units / upw;
  if (NW * upw != units || NW < 2 || NW > (upw == 2 ? 8 : 16) || (NW & (NW - 1))) return false;
  const PairLayout F = pair_layout<S>(X, Ycs, upw, C);
  if (F.Ux != units || F.Uy != NW || F.total > max_smem) return false;
  cf.kind = kKindLine;
  cf.full = false;
  cf.pair = true;
  cf.upw = upw;
  cf.ld = pair_ld(X);
  cf.NT = 32 * NW;
  cf.KX = kLineK;
  cf.C = C;
  cf.gstate = false;
  cf.Ycs = Ycs;
  cf.smem_bytes = (size_t)F.total;
  cf.grid_elems = 0;
  return true;
}

// Line family, any sizes: one lane per grid line; needs numX <= 256 and at
// most 16 warps of units per CTA.  Rows per CTA are a multiple of 4 when
// split, so every CTA's bulk copies start on a 16-byte boundary.
template <typename S>
bool line_generic_cfg(int X, int Y, int C, int max_smem, Config& cf) {
  if (X > 256) return false;
  const int Ycs = C == 1 ? Y : (int)round4(ceil_div(Y, C));
  if (C > 1 && (C - 1) * Ycs >= Y) return false;  // a CTA would own no row
  const LineLayout L16 = line_layout<S>(X, Ycs, 16);
  if (L16.Ux > 16 || L16.Uy > 16) return false;
  const int NT = std::max(64, 32 * pow2ceil(std::max(L16.Ux, L16.Uy)));
  const LineLayout L = line_layout<S>(X, Ycs, NT / 32);
  if (L.total > max_smem) return false;
  cf.kind = kKindLine;
  cf.full = false;
  cf.pair = false;
  cf.ld = line_ld(X);
  cf.NT = NT;
  cf.KX = kLineK;
  cf.C = C;
  cf.gstate = false;
  cf.Ycs = Ycs;
  cf.smem_bytes = (size_t)L.total;
  cf.grid_elems = 0;
  return true;
}

// Chunk family: any numX up to 512; the grid on chip over C CTAs, or (gstate)
// in HBM scratch when nothing fits.
template <typename S>
bool chunk_cfg(int X, int Y, int C, int max_smem, bool gstate, Config& cf) {
  const int Xp = std::max(8, pow2ceil(X));
  const int Ycs = ceil_div(Y, C);
  if (C > 1 && (C - 1) * Ycs >= Y) return false;
  const SmemLayout L = smem_layout<S>(Xp, X, Ycs, !gstate);
  if ((size_t)L.total * sizeof(S) > (size_t)max_smem) return false;
  cf.kind = kKindChunk;
  cf.full = false;
  cf.pair = false;
  cf.ld = 0;
  cf.KX = Xp <= 256 ? 8 : 16;
  cf.gstate = gstate;
  cf.C = C;
  cf.Ycs = Ycs;
  cf.smem_bytes = (size_t)L.total * sizeof(S);
  cf.grid_elems = L.grid_elems;
  const int cells = Ycs * Xp;
  cf.NT = cells >= 4096 ? 512 : (cells >= 1024 ? 256 : 128);
  if (cf.KX == 16) cf.NT = std::min(cf.NT, 256);
  return true;
}

// Built-in choice: the smallest cluster the line family fits in (paired
// kernel with two units per warp, then with one unit per warp -- numX == 32
// --, then full tiles, then any sizes), else the chunk family on chip, else
// the chunk family on HBM.
template <typename S>
Config default_config(int X, int Y, int max_smem) {
  Config cf;
  for (int C = 1; C <= kMaxCluster; C *= 2) {
    if (line_pair_cfg<S>(X, Y, C, max_smem, cf)) return cf;
    if (line_pair_cfg<S>(X, Y, C, max_smem, cf, 1)) return cf;  // numX == 32
    if (line_full_cfg<S>(X, Y, C, max_smem, cf)) return cf;
    if (line_generic_cfg<S>(X, Y, C, max_smem, cf)) return cf;
  }
  for (int C = 1; C <= kMaxCluster; C *= 2)
    if (chunk_cfg<S>(X, Y, C, max_smem, false, cf)) return cf;
  chunk_cfg<S>(X, Y, 1, max_smem, true, cf);
  return cf;
}

// Every configuration that can run an X x Y grid: the search space of the
// autotuner, in the order the built-in choice prefers them.  Splits thinner
// than 16 rows per CTA (line family) or 8 (chunk family) are left out: the
// cluster folds would cost more than the rows.
template <typename S>
std::vector<Config> enum_configs(int X, int Y, int max_smem) {
  std::vector<Config> v;
  Config cf;
  for (int C = 1; C <= kMaxCluster; C *= 2) {
    if (line_pair_cfg<S>(X, Y, C, max_smem, cf)) v.push_back(cf);
    if (line_pair_cfg<S>(X, Y, C, max_smem, cf, 1)) v.push_back(cf);
    if (line_full_cfg<S>(X, Y, C, max_smem, cf)) v.push_back(cf);
    if (line_generic_cfg<S>(X, Y, C, max_smem, cf) && (C == 1 || cf.Ycs >= 16)) v.push_back(cf);
  }
  for (int C = 1; C <= kMaxCluster; C *= 2)
    if (chunk_cfg<S>(X, Y, C, max_smem, false, cf) && (C == 1 || cf.Ycs >= 8)) v.push_back(cf);
  if (v.empty() && chunk_cfg<S>(X, Y, 1, max_smem, true, cf)) v.push_back(cf);
  if (v.empty()) v.push_back(default_config<S>(X, Y, max_smem));
  return v;
}

int family_of(const Config& c) {
  if (c.kind == kKindChunk) return LVC_FAMILY_CHUNK;
  if (c.pair) return c.upw == 1 ? LVC_FAMILY_LINE_PAIR1 : LVC_FAMILY_LINE_PAIR;
  return c.full ? LVC_FAMILY_LINE_FULL : LVC_FAMILY_LINE;
}

bool same_shape(const Config& a, const Config& b) {
  return family_of(a) == family_of(b) && a.C == b.C && a.gstate == b.gstate;
}

using TuneKey = std::tuple<int, int, int>;  // numX, numY, precision

template <typename S>
int precision_of() { return sizeof(S) == sizeof(double) ? LVC_F64 : LVC_F32_STATE; }

// The configuration of an X x Y grid: the context's tuned shape, else the
// built-in choice.
template <typename S>
Config choose_config(const futhark_context* ctx, int X, int Y) {
  auto it = ctx->shapes.find(TuneKey{X, Y, precision_of<S>()});
  if (it != ctx->shapes.end()) return it->second.cf;
  return default_config<S>(X, Y, ctx->max_smem);
}

template <typename S, typename PV>
int prepare_launch(futhark_context* ctx, Launch& L, int max_sms = 0) {
  RbFn<S, PV> fn = rollback_fn<S, PV>(L.kind, L.NT, L.KX, L.gstate, L.full, L.pair, L.upw);
  if (!fn) return set_error(ctx, FUTHARK_PROGRAM_ERROR, "no rollback kernel for this configuration");
  // Several launch classes may share one kernel instantiation with different
  // shared-memory sizes: allow the device maximum once for all of them.
  LVC_CUDA(ctx, cudaFuncSetAttribute((const void*)fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     ctx->max_smem));
  if (L.C > 8)
    LVC_CUDA(ctx, cudaFuncSetAttribute((const void*)fn,
                                       cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
  // max_sms < 0: one CTA (cluster) per work item instead of a persistent
  // grid, so the block scheduler shares SMs among concurrent launches
  const bool per_item = max_sms < 0;
  const int sms = (max_sms > 0 && max_sms < ctx->num_sms) ? max_sms : ctx->num_sms;
  int resident = 0;
  if (L.C == 1) {
    int per_sm = 0;
    LVC_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, L.NT, L.smem_bytes));
    resident = per_sm * sms;
    L.sm_per_cta = per_sm > 0 ? 1.0 / per_sm : 1.0;
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
    L.sm_per_cta = ncl > 0 ? (double)ctx->num_sms / ((double)ncl * L.C) : 1.0;
    resident = (int)((int64_t)ncl * sms / ctx->num_sms);
    if (resident < 1 && ncl > 0) resident = 1;
  }
  if (resident <= 0)
    return set_error(ctx, FUTHARK_PROGRAM_ERROR, "rollback configuration does not fit on the device");
  L.grid = (per_item ? L.n_items : std::min(L.n_items, resident)) * L.C;
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
  return cudaLaunchKernelEx(&cfg, rollback_fn<S, PV>(L.kind, L.NT, L.KX, L.gstate, L.full, L.pair, L.upw), a);
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
  int nonempty = 0;
  for (const Launch& L : P->launches) nonempty += L.n_items > 0;
  // Fork: launch j of the (largest-first) classes goes to stream j % n, so
  // the classes run side by side and the block scheduler fills the SMs one
  // class leaves idle with CTAs of the next.  Timed runs stay on one stream.
  const int nf = ev ? 1 : std::min(P->n_streams, nonempty);
  if (nf > 1) {
    if ((e = cudaEventRecord(P->ev_fork, s)) != cudaSuccess) return e;
    for (int j = 1; j < nf; j++)
      if ((e = cudaStreamWaitEvent(P->aux[j - 1], P->ev_fork, 0)) != cudaSuccess) return e;
  }
  int j = 0;
  for (size_t i = 0; i < P->launches.size(); i++) {
    const Launch& L = P->launches[i];
    if (L.n_items == 0) continue;
    const int si = nf > 1 ? j % nf : 0;
    j++;
    cudaStream_t ls = si == 0 ? s : P->aux[si - 1];
    if (ev && (e = cudaEventRecord(ev[2 * i], ls)) != cudaSuccess) return e;
    e = P->precision == LVC_F64 ? launch_rollback<double, double>(P, L, ls)
                                : launch_rollback<float, float>(P, L, ls);
    if (e != cudaSuccess) return e;
    if (ev && (e = cudaEventRecord(ev[2 * i + 1], ls)) != cudaSuccess) return e;
  }
  for (int k = 1; k < nf; k++) {
    if ((e = cudaEventRecord(P->ev_join[k - 1], P->aux[k - 1])) != cudaSuccess) return e;
    if ((e = cudaStreamWaitEvent(s, P->ev_join[k - 1], 0)) != cudaSuccess) return e;
  }
  return cudaSuccess;
}

void plan_release(lvc_plan* P) {
  if (!P) return;
  if (P->exec) cudaGraphExecDestroy(P->exec);
  if (P->graph) cudaGraphDestroy(P->graph);
  if (P->ev_fork) cudaEventDestroy(P->ev_fork);
  for (cudaEvent_t e : P->ev_join)
    if (e) cudaEventDestroy(e);
  void* bufs[] = {P->d_calibs, P->d_tabs, P->d_piv, P->d_out, P->d_rowstart, P->d_items, P->d_gstate, P->d_err};
  for (void* b : bufs) {
    if (!b) continue;
    if (P->pool) P->pool->release(b); else cudaFree(b);
  }
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
  P->cfgs.resize(n);
  P->row_start.assign(n + 1, 0);
  std::map<std::tuple<int, int, int, int, bool, bool, bool, int>, std::vector<std::pair<int64_t, Item>>> classes;
  std::map<std::tuple<int, int, int, int, bool, bool, bool, int>, Config> class_cfg;
  int64_t tab_off = 0, piv_off = 0, out_off = 0;
  for (int i = 0; i < n; i++) {
    const lvc_calibration& c = cs[i];
    if (int rc = validate(ctx, c, i)) return rc;
    const Config cf = choose_config<S>(ctx, c.numX, c.numY);
    P->cfgs[i] = cf;
    CalibDev& d = P->calibs[i];
    d.numX = c.numX;
    d.numY = c.numY;
    d.numT = c.numT;
    d.Xp = std::max(8, pow2ceil(c.numX));
    d.outer = c.outer;
    d.C = cf.C;
    d.kind = cf.kind;
    d.Ycs = cf.Ycs;
    d.ld = cf.ld;
    d.pad1 = 0;
    fill_scalars(d, c);
    d.tab = tab_off;
    tab_off += al2(tab_layout(c.numX, c.numY, c.numT, d.Xp, d.kind).total);
    d.piv = piv_off;
    piv_off += (piv_elems(c.numX, c.numY, c.numT, d.Xp, d.kind, d.ld) + 3) & ~int64_t(3);
    d.out = out_off;
    out_off += c.outer;
    P->row_start[i + 1] = P->row_start[i] + (int64_t)(c.numT > 1 ? c.numT - 1 : 0) * c.numY;
    const auto key = std::make_tuple(cf.kind, cf.NT, cf.KX, cf.C, cf.gstate, cf.full, cf.pair, cf.upw);
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
  std::vector<int64_t> class_work;
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
    L.pair = cf.pair;
    L.upw = cf.upw;
    L.NT = cf.NT;
    L.KX = cf.KX;
    L.C = cf.C;
    L.gstate = cf.gstate;
    L.item_off = (int)P->items.size();
    L.n_items = (int)v.size();
    L.smem_bytes = cf.smem_bytes;
    L.gstate_per_cta = cf.gstate ? cf.grid_elems : 0;
    int64_t work = 0;
    for (auto& e : v) {
      P->items.push_back(e.second);
      work += e.first;
    }
    class_work.push_back(work);
    L.work = work;
    if (L.n_items > 0) {
      if (int rc = prepare_launch<S, PV>(ctx, L, P->max_sms)) return rc;
      P->sms = std::max(P->sms, std::min<double>(L.grid * L.sm_per_cta, ctx->num_sms));
    } else {
      L.grid = 0;
    }
    L.gstate_off = gstate_off;
    if (L.gstate) gstate_off += (int64_t)L.grid * L.gstate_per_cta;
    P->launches.push_back(L);
  }
  P->gstate_elems = gstate_off;
  {  // largest class first: it starts first and sets the critical path
    std::vector<size_t> ord(P->launches.size());
    for (size_t i = 0; i < ord.size(); i++) ord[i] = i;
    std::stable_sort(ord.begin(), ord.end(), [&](size_t a, size_t b) { return class_work[a] > class_work[b]; });
    std::vector<Launch> sorted;
    for (size_t i : ord) sorted.push_back(P->launches[i]);
    P->launches.swap(sorted);
  }
  const int64_t rows = P->row_start[n];
  P->pivot_grid = (int)std::max<int64_t>(1, std::min<int64_t>((rows + 127) / 128, 64LL * ctx->num_sms));

  // device buffers
  auto dalloc = [&](void** dst, size_t bytes) -> int {
    if (P->pool) {
      *dst = P->pool->alloc(bytes);
      if (!*dst) return set_error(ctx, FUTHARK_OUT_OF_MEMORY, "device memory pool exhausted");
      return 0;
    }
    LVC_CUDA(ctx, cudaMalloc(dst, bytes));
    return 0;
  };
  if (int rc = dalloc((void**)&P->d_calibs, sizeof(CalibDev) * std::max(1, n))) return rc;
  if (int rc = dalloc((void**)&P->d_tabs, sizeof(double) * std::max<int64_t>(2, P->tab_elems))) return rc;
  if (int rc = dalloc(&P->d_piv, sizeof(PV) * std::max<int64_t>(4, P->piv_elems))) return rc;
  if (int rc = dalloc((void**)&P->d_out, sizeof(double) * std::max<int64_t>(1, P->nprices))) return rc;
  if (int rc = dalloc((void**)&P->d_rowstart, sizeof(int64_t) * (n + 1))) return rc;
  if (int rc = dalloc((void**)&P->d_items, sizeof(Item) * std::max<size_t>(1, P->items.size()))) return rc;
  if (P->gstate_elems > 0)
    if (int rc = dalloc(&P->d_gstate, sizeof(S) * P->gstate_elems)) return rc;
  if (int rc = dalloc((void**)&P->d_err, sizeof(int))) return rc;
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
  if (!P->use_graph) return 0;

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
                    lvc_plan** out, DevicePool* pool = nullptr, bool use_graph = true,
                    int max_sms = 0) {
  if (!ctx->ok) return set_error(ctx, FUTHARK_PROGRAM_ERROR, "context has no usable CUDA device");
  if (n < 0 || (n > 0 && !cs)) return set_error(ctx, FUTHARK_PROGRAM_ERROR, "bad calibration list");
  if (precision != LVC_F64 && precision != LVC_F32_STATE)
    return set_error(ctx, FUTHARK_PROGRAM_ERROR, "unknown precision");
  LVC_CUDA(ctx, cudaSetDevice(ctx->device));
  lvc_plan* P = new lvc_plan();
  P->precision = precision;
  P->pool = pool;
  P->use_graph = use_graph;
  P->max_sms = max_sms;
  P->shapes_gen = ctx->shapes_gen;
  if (use_graph && max_sms == 0) {  // batch plans follow the context's tuning
    P->max_sms = grid_mode(ctx->tuning, precision) == 1 ? -1 : 0;
    P->n_streams = ctx->tuning.streams;
    for (int k = 0; k < kMaxAux; k++) P->aux[k] = ctx->aux[k];
    LVC_CUDA(ctx, cudaEventCreateWithFlags(&P->ev_fork, cudaEventDisableTiming));
    for (int k = 0; k + 1 < P->n_streams; k++)
      LVC_CUDA(ctx, cudaEventCreateWithFlags(&P->ev_join[k], cudaEventDisableTiming));
  }
  const int rc = precision == LVC_F64 ? plan_build<double, double>(ctx, cs, n, P)
                                      : plan_build<float, float>(ctx, cs, n, P);
  if (rc) {
    plan_release(P);
    return rc;
  }
  *out = P;
  return 0;
}

// One run of a plan on stream s: the captured graph when there is one.
cudaError_t plan_launch(lvc_plan* P, cudaStream_t s) {
  if (P->exec) return cudaGraphLaunch(P->exec, s);
  return plan_enqueue(P, s, nullptr);
}

// Device memory of the generated API's arrays comes from the context's pool:
// a freed array's block serves the next one, so an entry-point call does not
// reach cudaMalloc/cudaFree (cudaFree synchronises the whole device and its
// cost varies from call to call).  Called with ctx->mu held.
void* arr_alloc(futhark_context* ctx, size_t bytes) {
  if (!ctx->pool) ctx->pool = new DevicePool();
  return ctx->pool->alloc(bytes);
}
void arr_free(futhark_context* ctx, void* p) {
  if (ctx->pool) ctx->pool->release(p);
}

int check_device_error(futhark_context* ctx, lvc_plan* P) {
  int h = 0;
  LVC_CUDA(ctx, cudaMemcpyAsync(&h, P->d_err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  LVC_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (h == 3) return set_error(ctx, FUTHARK_PROGRAM_ERROR, "rollback kernel: a bounded wait for a bulk copy timed out");
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
    // rebuilt when the sizes change, or the tuning table (the shape) did
    if (o.outer != c.outer || o.numX != c.numX || o.numY != c.numY || o.numT != c.numT ||
        P->shapes_gen != ctx->shapes_gen) {
      LVC_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
      plan_release(P);
      P = ctx->entry_plan = nullptr;
    }
  }
  if (!P) {
    if (!ctx->pool) ctx->pool = new DevicePool();
    if (int rc = plan_new_locked(ctx, &c, 1, LVC_F64, &P, ctx->pool, /*use_graph=*/false)) return rc;
    ctx->entry_plan = P;
  } else if (int rc = set_params_locked(ctx, P, &c, 1)) {
    return rc;
  }
  LVC_CUDA(ctx, plan_launch(P, ctx->stream));
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
int futhark_context_config_set_tuning_param(struct futhark_context_config* cfg, const char* param_name,
                                            size_t new_value) {
  if (!cfg) return 1;
  return set_tuning(cfg->tuning, param_name, new_value);
}
int futhark_get_tuning_param_count(void) { return kNumTuning; }
const char* futhark_get_tuning_param_name(int i) {
  return (i >= 0 && i < kNumTuning) ? kTuningNames[i] : nullptr;
}
const char* futhark_get_tuning_param_class(int i) {
  return (i >= 0 && i < kNumTuning) ? kTuningClasses[i] : nullptr;
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
  for (int k = 0; k < kMaxAux; k++)
    if ((e = cudaStreamCreateWithFlags(&ctx->aux[k], cudaStreamNonBlocking)) != cudaSuccess) {
      ctx->error = std::string("cannot create stream: ") + cudaGetErrorString(e);
      return ctx;
    }
  if (cfg) ctx->tuning = cfg->tuning;
  ctx->ok = true;
  return ctx;
}

void futhark_context_free(struct futhark_context* ctx) {
  if (!ctx) return;
  if (ctx->ok) {
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    plan_release(ctx->entry_plan);
    delete ctx->pool;
    cudaStreamDestroy(ctx->stream);
    cudaStreamDestroy(ctx->capture);
    for (cudaStream_t a : ctx->aux)
      if (a) cudaStreamDestroy(a);
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
  // blocks still held by the caller's plans stay; every free one is returned
  if (ctx->pool) ctx->pool->trim();
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
    if (!(a->data = static_cast<T*>(arr_alloc(ctx, a->bytes)))) {                                \
      ctx->error = "out of device memory";                                                       \
      delete a;                                                                                  \
      return nullptr;                                                                            \
    }                                                                                            \
    if (dim0 > 0 && data &&                                                                      \
        cudaMemcpyAsync(a->data, data, sizeof(T) * dim0, cudaMemcpyHostToDevice, ctx->stream) != \
            cudaSuccess) {                                                                       \
      arr_free(ctx, a->data);                                                                    \
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
    arr_free(ctx, arr->data);                                                                    \
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
  if (!(a->data = static_cast<double*>(arr_alloc(ctx, a->bytes)))) {
    delete a;
    return set_error(ctx, FUTHARK_OUT_OF_MEMORY, "out of device memory");
  }
  cudaError_t e;
  if (outer > 0 && (e = cudaMemcpyAsync(a->data, ctx->entry_plan->d_out, sizeof(double) * outer,
                                        cudaMemcpyDeviceToDevice, ctx->stream)) != cudaSuccess) {
    arr_free(ctx, a->data);
    delete a;
    return cuda_fail(ctx, e, "cudaMemcpyAsync");
  }
  if (int rc = check_device_error(ctx, ctx->entry_plan)) {
    arr_free(ctx, a->data);
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
  if (!(a->data = static_cast<float*>(arr_alloc(ctx, a->bytes)))) {
    delete a;
    return set_error(ctx, FUTHARK_OUT_OF_MEMORY, "out of device memory");
  }
  if (outer > 0) {
    lvc_to_f32_kernel<<<(outer + 255) / 256, 256, 0, ctx->stream>>>(ctx->entry_plan->d_out, a->data,
                                                                     outer);
    cudaError_t e;
    if ((e = cudaGetLastError()) != cudaSuccess) {
      arr_free(ctx, a->data);
      delete a;
      return cuda_fail(ctx, e, "lvc_to_f32_kernel");
    }
  }
  if (int rc = check_device_error(ctx, ctx->entry_plan)) {
    arr_free(ctx, a->data);
    delete a;
    return rc;
  }
  *out0 = a;
  return 0;
}

int lvc_plan_new(struct futhark_context* ctx, const struct lvc_calibration* calibs, int32_t n,
                 int32_t precision, struct lvc_plan** plan) {
  std::lock_guard<std::mutex> g(ctx->mu);
  if (ctx->ok && !ctx->pool) ctx->pool = new DevicePool();
  return plan_new_locked(ctx, calibs, n, precision, plan, ctx->pool);
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
  LVC_CUDA(ctx, plan_launch(plan, ctx->stream));
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
  for (int i = 0; i < iters; i++) LVC_CUDA(ctx, plan_launch(plan, ctx->stream));
  LVC_CUDA(ctx, cudaEventRecord(b, ctx->stream));
  LVC_CUDA(ctx, cudaEventSynchronize(b));
  float ms = 0.f;
  LVC_CUDA(ctx, cudaEventElapsedTime(&ms, a, b));
  *ms_per_run = ms / iters;
  // the rollback launches alone, with events between the kernels
  std::vector<cudaEvent_t> ev(2 * plan->launches.size());
  for (auto& x : ev) LVC_CUDA(ctx, cudaEventCreate(&x));
  double roll = 0.0;
  for (Launch& L : plan->launches) L.ms = 0.0;
  for (int i = 0; i < iters; i++) {
    cudaError_t e = plan_enqueue(plan, ctx->stream, ev.data());
    if (e != cudaSuccess) return cuda_fail(ctx, e, "plan_enqueue");
    LVC_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    for (size_t l = 0; l < plan->launches.size(); l++) {
      if (plan->launches[l].n_items == 0) continue;
      float t = 0.f;
      LVC_CUDA(ctx, cudaEventElapsedTime(&t, ev[2 * l], ev[2 * l + 1]));
      roll += t;
      plan->launches[l].ms += t / iters;
    }
  }
  plan->rollback_ms = roll / iters;
  for (auto& x : ev) cudaEventDestroy(x);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return check_device_error(ctx, plan);
}

double lvc_plan_rollback_ms(const struct lvc_plan* plan) { return plan ? plan->rollback_ms : 0.0; }

int32_t lvc_plan_num_classes(const struct lvc_plan* plan) { return plan ? (int32_t)plan->launches.size() : 0; }

int lvc_plan_launch_info(const struct lvc_plan* plan, int32_t i, struct lvc_launch_info* out) {
  if (!plan || !out || i < 0 || i >= (int32_t)plan->launches.size()) return -1;
  const Launch& L = plan->launches[i];
  Config c{};
  c.kind = L.kind;
  c.full = L.full;
  c.pair = L.pair;
  c.upw = L.upw;
  out->family = family_of(c);
  out->cluster = L.C;
  out->threads = L.NT;
  out->items = L.n_items;
  out->cell_steps = L.work;
  out->ms = L.ms;
  return 0;
}

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

int lvc_context_set_tuning_param(struct futhark_context* ctx, const char* param_name, size_t new_value) {
  std::lock_guard<std::mutex> g(ctx->mu);
  if (set_tuning(ctx->tuning, param_name, new_value))
    return set_error(ctx, FUTHARK_PROGRAM_ERROR,
                     std::string("unknown tuning parameter or value: ") + (param_name ? param_name : "(null)"));
  return 0;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Shape autotuner.  For every grid class (numX, numY) of a workload it times
// each configuration that can run the class -- kernel family, cluster size
// and the CTA shape that follows from them -- on the class's own number of
// strike instances for a few time steps, and keeps the fastest in the
// context's tuning table, which every plan, entry point and server built
// from the context then uses.  The table is written and read as a tuning
// file of `name=value` lines, the form of Futhark's own tuning files.
// ---------------------------------------------------------------------------
namespace {

const char* family_name(int fam, bool gstate) {
  if (fam == LVC_FAMILY_LINE_PAIR1) return "line_pair1";
  if (fam == LVC_FAMILY_LINE_PAIR) return "line_pair";
  if (fam == LVC_FAMILY_LINE_FULL) return "line_full";
  if (fam == LVC_FAMILY_LINE) return "line";
  return gstate ? "chunk_hbm" : "chunk";
}

void to_shape(const Config& c, lvc_shape* o) {
  o->family = family_of(c);
  o->cluster = c.C;
  o->threads = c.NT;
  o->rows_per_cta = c.Ycs;
  o->smem_bytes = (int32_t)c.smem_bytes;
  o->hbm_state = c.gstate ? 1 : 0;
}

int check_grid(futhark_context* ctx, int X, int Y, int precision) {
  if (precision != LVC_F64 && precision != LVC_F32_STATE)
    return set_error(ctx, FUTHARK_PROGRAM_ERROR, "unknown precision");
  if (X < 3 || Y < 3 || X > kMaxNumX || Y > kMaxNumY)
    return set_error(ctx, FUTHARK_PROGRAM_ERROR, "grid size out of range");
  return 0;
}

std::vector<Config> candidates(const futhark_context* ctx, int X, int Y, int precision) {
  return precision == LVC_F64 ? enum_configs<double>(X, Y, ctx->max_smem)
                              : enum_configs<float>(X, Y, ctx->max_smem);
}

Config builtin(const futhark_context* ctx, int X, int Y, int precision) {
  return precision == LVC_F64 ? default_config<double>(X, Y, ctx->max_smem)
                              : default_config<float>(X, Y, ctx->max_smem);
}

// Microseconds per time step of the rollback launch of calibration c under
// the context's current table (median of `reps` timed runs after one warm-up).
constexpr double kTuneMargin = 1.03;  // a shape replaces the built-in one only when 3% faster

int probe_us_per_step(futhark_context* ctx, const lvc_calibration& c, int precision, int reps, double* us) {
  if (!ctx->pool) ctx->pool = new DevicePool();
  lvc_plan* P = nullptr;
  const int max_sms = grid_mode(ctx->tuning, precision) == 1 ? -1 : 0;
  if (int rc = plan_new_locked(ctx, &c, 1, precision, &P, ctx->pool, /*use_graph=*/false, max_sms)) return rc;
  std::vector<cudaEvent_t> ev(2 * P->launches.size(), nullptr);
  for (auto& x : ev) {
    cudaError_t e = cudaEventCreate(&x);
    if (e != cudaSuccess) {
      for (auto& y : ev)
        if (y) cudaEventDestroy(y);
      plan_release(P);
      return cuda_fail(ctx, e, "cudaEventCreate");
    }
  }
  std::vector<double> t;
  int rc = 0;
  for (int r = 0; r <= reps && !rc; r++) {
    cudaError_t e = plan_enqueue(P, ctx->stream, ev.data());
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
      rc = cuda_fail(ctx, e, "autotune probe");
      break;
    }
    double ms = 0.0;
    for (size_t l = 0; l < P->launches.size(); l++) {
      if (P->launches[l].n_items == 0) continue;
      float x = 0.f;
      cudaEventElapsedTime(&x, ev[2 * l], ev[2 * l + 1]);
      ms += x;
    }
    if (r > 0) t.push_back(ms);
  }
  if (!rc) rc = check_device_error(ctx, P);
  for (auto& x : ev) cudaEventDestroy(x);
  plan_release(P);
  if (rc) return rc;
  std::sort(t.begin(), t.end());
  *us = t.empty() ? 0.0 : 1e3 * t[t.size() / 2] / std::max(1, c.numT - 1);
  return 0;
}

}  // namespace

extern "C" {

int lvc_shape_candidates(struct futhark_context* ctx, int32_t numX, int32_t numY, int32_t precision,
                         struct lvc_shape* out, int32_t max, int32_t* count) {
  std::lock_guard<std::mutex> g(ctx->mu);
  if (int rc = check_grid(ctx, numX, numY, precision)) return rc;
  const std::vector<Config> v = candidates(ctx, numX, numY, precision);
  for (int i = 0; i < (int)v.size() && i < max; i++) to_shape(v[i], &out[i]);
  if (count) *count = (int32_t)v.size();
  return 0;
}

int lvc_tuning_set(struct futhark_context* ctx, int32_t numX, int32_t numY, int32_t precision,
                   const struct lvc_shape* shape) {
  std::lock_guard<std::mutex> g(ctx->mu);
  if (int rc = check_grid(ctx, numX, numY, precision)) return rc;
  const TuneKey key{numX, numY, precision};
  if (!shape) {
    ctx->shapes.erase(key);
    ctx->shapes_gen++;
    return 0;
  }
  for (const Config& c : candidates(ctx, numX, numY, precision)) {
    if (family_of(c) == shape->family && c.C == shape->cluster && (c.gstate ? 1 : 0) == shape->hbm_state) {
      TunedShape t;
      t.cf = c;
      t.tuned = true;
      ctx->shapes[key] = t;
      ctx->shapes_gen++;
      return 0;
    }
  }
  return set_error(ctx, FUTHARK_PROGRAM_ERROR, "no such shape for this grid size on this device");
}

int lvc_tuning_get(struct futhark_context* ctx, int32_t numX, int32_t numY, int32_t precision,
                   struct lvc_tuning_entry* out) {
  std::lock_guard<std::mutex> g(ctx->mu);
  if (int rc = check_grid(ctx, numX, numY, precision)) return rc;
  *out = lvc_tuning_entry{};
  out->numX = numX;
  out->numY = numY;
  out->precision = precision;
  auto it = ctx->shapes.find(TuneKey{numX, numY, precision});
  if (it != ctx->shapes.end()) {
    to_shape(it->second.cf, &out->shape);
    out->tuned = it->second.tuned ? 1 : 0;
    out->us_per_step_default = it->second.us_default;
    out->us_per_step_best = it->second.us_best;
  } else {
    to_shape(builtin(ctx, numX, numY, precision), &out->shape);
  }
  return 0;
}

int lvc_plan_shape(const struct lvc_plan* plan, int32_t calib, struct lvc_shape* out) {
  if (!plan || !out || calib < 0 || calib >= plan->ncal) return FUTHARK_PROGRAM_ERROR;
  to_shape(plan->cfgs[calib], out);
  return 0;
}

int32_t lvc_tuning_entries(struct futhark_context* ctx, struct lvc_tuning_entry* out, int32_t max) {
  std::lock_guard<std::mutex> g(ctx->mu);
  int32_t n = 0;
  for (const auto& kv : ctx->shapes) {
    if (out && n < max) {
      lvc_tuning_entry& e = out[n];
      e = lvc_tuning_entry{};
      e.numX = std::get<0>(kv.first);
      e.numY = std::get<1>(kv.first);
      e.precision = std::get<2>(kv.first);
      e.tuned = kv.second.tuned ? 1 : 0;
      to_shape(kv.second.cf, &e.shape);
      e.us_per_step_default = kv.second.us_default;
      e.us_per_step_best = kv.second.us_best;
    }
    n++;
  }
  return n;
}

int lvc_autotune(struct futhark_context* ctx, const struct lvc_calibration* calibs, int32_t n,
                 int32_t precision, int32_t probe_steps) {
  std::lock_guard<std::mutex> g(ctx->mu);
  if (!ctx->ok) return set_error(ctx, FUTHARK_PROGRAM_ERROR, "context has no usable CUDA device");
  if (precision != LVC_F64 && precision != LVC_F32_STATE)
    return set_error(ctx, FUTHARK_PROGRAM_ERROR, "unknown precision");
  if (n < 0 || (n > 0 && !calibs)) return set_error(ctx, FUTHARK_PROGRAM_ERROR, "bad calibration list");
  LVC_CUDA(ctx, cudaSetDevice(ctx->device));
  if (probe_steps <= 0) probe_steps = 8;
  // grid classes: instance count and a representative calibration
  std::map<std::pair<int, int>, std::pair<int64_t, lvc_calibration>> classes;
  for (int i = 0; i < n; i++) {
    if (int rc = validate(ctx, calibs[i], i)) return rc;
    if (calibs[i].outer == 0 || calibs[i].numT < 2) continue;
    auto& e = classes[{calibs[i].numX, calibs[i].numY}];
    if (e.first == 0) e.second = calibs[i];
    e.first += calibs[i].outer;
  }
  for (const auto& kv : classes) {
    const int X = kv.first.first, Y = kv.first.second;
    const TuneKey key{X, Y, precision};
    const std::vector<Config> cands = candidates(ctx, X, Y, precision);
    const Config def = builtin(ctx, X, Y, precision);
    lvc_calibration probe = kv.second.second;
    probe.outer = (int32_t)std::min<int64_t>(kv.second.first, 1 << 14);
    probe.numT = probe_steps + 1;
    TunedShape best;
    best.cf = def;
    best.tuned = true;
    double best_us = 0.0, def_us = 0.0;
    bool any = false;
    for (const Config& c : cands) {
      TunedShape t;
      t.cf = c;
      t.tuned = true;
      ctx->shapes[key] = t;
      double us = 0.0;
      if (probe_us_per_step(ctx, probe, precision, 3, &us)) {
        ctx->error.clear();  // a shape that cannot run here is skipped
        continue;
      }
      if (same_shape(c, def)) def_us = us;
      // the built-in shape is kept unless another wins by a clear margin: a
      // class's probe runs alone, while in a plan it overlaps other classes
      const double margin = same_shape(c, def) ? 1.0 / kTuneMargin : (same_shape(best.cf, def) ? kTuneMargin : 1.0);
      if (!any || us * margin < best_us) {
        best.cf = c;
        best_us = us;
        any = true;
      }
    }
    if (any && same_shape(best.cf, def) && def_us > 0.0) best_us = def_us;
    if (!any) {
      ctx->shapes.erase(key);
      ctx->shapes_gen++;
      return set_error(ctx, FUTHARK_PROGRAM_ERROR, "autotune: no shape ran for a grid class");
    }
    best.us_best = best_us;
    best.us_default = def_us;
    ctx->shapes[key] = best;
  }
  ctx->shapes_gen++;
  return 0;
}

int lvc_autotune_plan(struct futhark_context* ctx, const struct lvc_calibration* calibs, int32_t n,
                      int32_t precision, int32_t max_steps, int32_t* grid, int32_t* streams, double* ms) {
  std::lock_guard<std::mutex> g(ctx->mu);
  if (!ctx->ok) return set_error(ctx, FUTHARK_PROGRAM_ERROR, "context has no usable CUDA device");
  if (precision != LVC_F64 && precision != LVC_F32_STATE)
    return set_error(ctx, FUTHARK_PROGRAM_ERROR, "unknown precision");
  if (n <= 0 || !calibs) return set_error(ctx, FUTHARK_PROGRAM_ERROR, "bad calibration list");
  LVC_CUDA(ctx, cudaSetDevice(ctx->device));
  if (max_steps <= 0) max_steps = 32;
  // the workload with its time lines capped: the same classes, instances and
  // shapes, a fraction of the steps
  std::vector<lvc_calibration> probe(calibs, calibs + n);
  for (auto& c : probe) c.numT = std::min(c.numT, max_steps + 1);
  const TuningParams keep = ctx->tuning;
  TuningParams best = keep;
  double best_ms = -1.0;
  cudaEvent_t e0, e1;
  LVC_CUDA(ctx, cudaEventCreate(&e0));
  LVC_CUDA(ctx, cudaEventCreate(&e1));
  // the capped plan under the context's current tuning: the faster of two
  // runs after a warm-up run
  auto time_plan = [&](double* t) -> int {
    lvc_plan* P = nullptr;
    if (int rc = plan_new_locked(ctx, probe.data(), n, precision, &P)) return rc;
    int rc = 0;
    *t = 1e30;
    for (int r = 0; r < 3 && !rc; r++) {
      cudaError_t e = cudaEventRecord(e0, ctx->stream);
      if (e == cudaSuccess) e = plan_launch(P, ctx->stream);
      if (e == cudaSuccess) e = cudaEventRecord(e1, ctx->stream);
      if (e == cudaSuccess) e = cudaEventSynchronize(e1);
      float x = 0.f;
      if (e == cudaSuccess) e = cudaEventElapsedTime(&x, e0, e1);
      if (e != cudaSuccess) rc = cuda_fail(ctx, e, "autotune plan run");
      if (r > 0) *t = std::min(*t, (double)x);  // the first run warms up
    }
    if (!rc) rc = check_device_error(ctx, P);
    plan_release(P);
    return rc;
  };
  int rc = 0;
  for (int gm = 0; gm <= 1 && !rc; gm++) {
    for (int st : {2, 4}) {
      ctx->tuning.grid = gm;
      ctx->tuning.streams = st;
      double t = 0.0;
      if ((rc = time_plan(&t))) break;
      if (best_ms < 0 || t < best_ms) {
        best_ms = t;
        best = ctx->tuning;
      }
    }
  }
  ctx->tuning = rc ? keep : best;
  // A class shape that the per-class autotuner changed won alone, in a probe
  // of that class only; in the plan it overlaps the other classes.  Keep the
  // change only if the whole plan is faster with it than with the built-in
  // shape of that class.
  if (!rc) {
    std::set<TuneKey> changed;
    for (int i = 0; i < n; i++) {
      const TuneKey key{probe[i].numX, probe[i].numY, precision};
      auto it = ctx->shapes.find(key);
      if (it != ctx->shapes.end() && !same_shape(it->second.cf, builtin(ctx, probe[i].numX, probe[i].numY, precision)))
        changed.insert(key);
    }
    for (const TuneKey& key : changed) {
      const TunedShape tuned = ctx->shapes[key];
      TunedShape def = tuned;
      def.cf = builtin(ctx, std::get<0>(key), std::get<1>(key), precision);
      ctx->shapes[key] = def;
      ctx->shapes_gen++;
      double t = 0.0;
      if ((rc = time_plan(&t))) {
        ctx->shapes[key] = tuned;
        ctx->shapes_gen++;
        break;
      }
      if (t < best_ms) {
        best_ms = t;  // the built-in shape stays
      } else {
        ctx->shapes[key] = tuned;
        ctx->shapes_gen++;
      }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) {
    ctx->tuning = keep;
    return rc;
  }
  if (grid) *grid = best.grid;
  if (streams) *streams = best.streams;
  if (ms) *ms = best_ms;
  return 0;
}

int lvc_tuning_save(struct futhark_context* ctx, const char* path) {
  std::lock_guard<std::mutex> g(ctx->mu);
  FILE* f = path ? fopen(path, "w") : nullptr;
  if (!f) return set_error(ctx, FUTHARK_PROGRAM_ERROR, std::string("cannot write tuning file ") + (path ? path : ""));
  fprintf(f, "lvc.streams=%d\nlvc.grid=%d\n", ctx->tuning.streams, ctx->tuning.grid);
  for (const auto& kv : ctx->shapes)
    fprintf(f, "lvc.shape.%s.%dx%d=%s,%d\n", std::get<2>(kv.first) == LVC_F64 ? "f64" : "f32state",
            std::get<0>(kv.first), std::get<1>(kv.first),
            family_name(family_of(kv.second.cf), kv.second.cf.gstate), kv.second.cf.C);
  fclose(f);
  return 0;
}

int lvc_tuning_load(struct futhark_context* ctx, const char* path) {
  FILE* f = path ? fopen(path, "r") : nullptr;
  if (!f) {
    std::lock_guard<std::mutex> g(ctx->mu);
    return set_error(ctx, FUTHARK_PROGRAM_ERROR, std::string("cannot read tuning file ") + (path ? path : ""));
  }
  char line[256];
  int lineno = 0, rc = 0;
  while (!rc && fgets(line, sizeof line, f)) {
    lineno++;
    char* nl = strpbrk(line, "\r\n");
    if (nl) *nl = 0;
    if (!line[0] || line[0] == '#') continue;
    char prec[16], fam[16];
    int X = 0, Y = 0, C = 0;
    unsigned long v = 0;
    char name[128];
    if (sscanf(line, "lvc.shape.%15[a-z0-9].%dx%d=%15[a-z_0-9],%d", prec, &X, &Y, fam, &C) == 5) {
      lvc_shape sh{};
      sh.cluster = C;
      const std::string fs(fam);
      sh.family = fs == "line_pair1"  ? LVC_FAMILY_LINE_PAIR1
                  : fs == "line_pair" ? LVC_FAMILY_LINE_PAIR
                  : fs == "line_full" ? LVC_FAMILY_LINE_FULL
                  : fs == "line"      ? LVC_FAMILY_LINE
                                      : LVC_FAMILY_CHUNK;
      sh.hbm_state = fs == "chunk_hbm" ? 1 : 0;
      const bool known = fs == "line_pair1" || fs == "line_pair" || fs == "line_full" || fs == "line" || fs == "chunk" || fs == "chunk_hbm";
      const int p = !strcmp(prec, "f64") ? LVC_F64 : !strcmp(prec, "f32state") ? LVC_F32_STATE : -1;
      if (!known || p < 0) rc = 1;
      else rc = lvc_tuning_set(ctx, X, Y, p, &sh);
    } else if (sscanf(line, "%127[a-z.]=%lu", name, &v) == 2) {
      std::lock_guard<std::mutex> g(ctx->mu);
      rc = set_tuning(ctx->tuning, name, v) ? 1 : 0;
    } else {
      rc = 1;
    }
  }
  fclose(f);
  if (rc) {
    std::lock_guard<std::mutex> g(ctx->mu);
    char buf[160];
    snprintf(buf, sizeof buf, "tuning file %s: line %d not understood or not valid on this device", path, lineno);
    return set_error(ctx, FUTHARK_PROGRAM_ERROR, buf);
  }
  return 0;
}

int lvc_probe_peaks(struct futhark_context* ctx, double* fp64_tflops, double* smem_gbs) {
  std::lock_guard<std::mutex> g(ctx->mu);
  if (!ctx->ok) return set_error(ctx, FUTHARK_PROGRAM_ERROR, "context has no usable CUDA device");
  LVC_CUDA(ctx, cudaSetDevice(ctx->device));
  // released on every return, the early error returns of LVC_CUDA included
  struct Probe {
    void* scratch = nullptr;
    cudaEvent_t a = nullptr, b = nullptr;
    ~Probe() {
      if (a) cudaEventDestroy(a);
      if (b) cudaEventDestroy(b);
      if (scratch) cudaFree(scratch);
    }
  } pr;
  LVC_CUDA(ctx, cudaMalloc(&pr.scratch, 1 << 20));
  LVC_CUDA(ctx, cudaEventCreate(&pr.a));
  LVC_CUDA(ctx, cudaEventCreate(&pr.b));
  void* const scratch = pr.scratch;
  const cudaEvent_t a = pr.a, b = pr.b;
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

// The scratch carve-up of one call: calibration record, error flag, row
// table, work list, operator tables and pivot rows, each on a 256-byte boundary.
struct NoallocCarve {
  size_t o_calib, o_err, o_rows, o_items, o_tabs, o_piv, need;
};
NoallocCarve noalloc_carve(const Config& cf, int outer, int numX, int numY, int numT) {
  const int Xp = std::max(8, pow2ceil(numX));
  const int64_t tab_elems = al2(tab_layout(numX, numY, numT, Xp, cf.kind).total);
  const int64_t piv_n = (piv_elems(numX, numY, numT, Xp, cf.kind, cf.ld) + 3) & ~int64_t(3);
  NoallocCarve c;
  c.o_calib = 0;
  c.o_err = up256(c.o_calib + sizeof(CalibDev));
  c.o_rows = up256(c.o_err + sizeof(int));
  c.o_items = up256(c.o_rows + 2 * sizeof(int64_t));
  c.o_tabs = up256(c.o_items + sizeof(Item) * (size_t)std::max(1, outer));
  c.o_piv = up256(c.o_tabs + sizeof(double) * (size_t)tab_elems);
  c.need = c.o_piv + sizeof(double) * (size_t)piv_n;
  return c;
}

extern "C" int64_t lvc_entry_main_f64_noalloc_bytes(struct futhark_context* ctx, const int32_t outer,
                                                    const int32_t numX, const int32_t numY, const int32_t numT) {
  if (!ctx) return -1;
  std::lock_guard<std::mutex> g(ctx->mu);
  if (outer < 0 || numX < 3 || numY < 3 || numT < 1 || numX > kMaxNumX || numY > kMaxNumY) return -1;
  const Config cf = choose_config<double>(ctx, numX, numY);
  if (cf.gstate) return -1;
  return (int64_t)noalloc_carve(cf, outer, numX, numY, numT).need;
}

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

  const Config cf = choose_config<double>(ctx, numX, numY);
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
  d.ld = cf.ld;
  fill_scalars(d, c);
  d.tab = 0;
  d.piv = 0;
  d.out = 0;
  const NoallocCarve cv = noalloc_carve(cf, outer, numX, numY, numT);
  const size_t o_calib = cv.o_calib, o_err = cv.o_err, o_rows = cv.o_rows, o_items = cv.o_items,
               o_tabs = cv.o_tabs, o_piv = cv.o_piv, need = cv.need;
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
    L.pair = cf.pair;
    L.upw = cf.upw;
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
    LVC_CUDA(ctx, cudaLaunchKernelEx(&cfg, rollback_fn<double, double>(L.kind, L.NT, L.KX, false, L.full, L.pair, L.upw), a));
  }
  int h = 0;
  LVC_CUDA(ctx, cudaMemcpyAsync(&h, d_err, sizeof(int), cudaMemcpyDeviceToHost, s));
  LVC_CUDA(ctx, cudaStreamSynchronize(s));
  if (h == 3) return set_error(ctx, FUTHARK_PROGRAM_ERROR, "rollback kernel: a bounded wait for a bulk copy timed out");
  if (h) return set_error(ctx, FUTHARK_PROGRAM_ERROR, "rollback kernel rejected a work item");
  return 0;
}

// ---------------------------------------------------------------------------
// Serving runtime: continuous batching of calibration requests.
//
// A scheduler thread owns a private context on the caller's device, a device
// memory pool capped at the HBM budget, and a set of streams.  Pending
// requests are admitted in FIFO order as batches whenever (a) a stream is
// free, (b) the in-flight request count is below its cap and (c) the batch's
// tables and pivots fit in what is left of the HBM budget.  A batch launches
// one CTA (or cluster) per strike instance, each holding its grid in shared
// memory for all its time steps; the block scheduler hands SMs -- i.e. their
// shared memory -- to the waiting CTAs of all in-flight batches as running
// instances finish, so requests that arrive while others are on the GPU start
// as soon as memory and SMs free up and their work overlaps.  Each instance
// runs the same kernels as every other entry point, so a price does not
// depend on what ran beside it.
// ---------------------------------------------------------------------------
namespace {

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct SrvRequest {
  uint64_t ticket = 0;
  lvc_calibration c{};
  double work = 0;  // option-cell-steps: the admission order's size estimate
  double t_submit = 0, t_done = 0;
  std::vector<double> prices;
  int status = 0;  // 0 pending / running, 1 done, 2 failed
  std::string error;
};

struct SrvBatch {
  std::vector<SrvRequest*> reqs;
  lvc_plan* plan = nullptr;
  bool cached = false;  // a one-request plan that goes back to the plan cache
  int stream = -1;
  cudaEvent_t done = nullptr;
  double sms = 0;
  double t_launch = 0;
};

}  // namespace

struct lvc_server {
  futhark_context* user_ctx = nullptr;
  futhark_context sctx;  // private context: device properties, upload stream, errors
  lvc_server_config cfg{};
  DevicePool pool;
  std::vector<cudaStream_t> streams;
  std::vector<bool> stream_busy;
  std::vector<bool> stream_high;  // created at the device's greatest priority: small batches go there
  std::vector<double*> pinned;  // per stream: staging for prices and the error flag
  std::vector<int64_t> pinned_cap;
  std::vector<double*> pinned_retired;  // outgrown staging, freed with the server (cudaFreeHost synchronises)
  int32_t max_batch_configured = 0;     // cfg.max_batch_requests as given; restored after a back-off
  // one-request plans kept for reuse, keyed by sizes (outer, numX, numY, numT);
  // idle ones hold pool memory and are evicted when admission needs it
  std::map<std::tuple<int, int, int, int>, std::vector<lvc_plan*>> plan_cache;
  std::deque<std::pair<std::tuple<int, int, int, int>, lvc_plan*>> plan_lru;  // idle plans, oldest first
  int64_t plans_reused = 0;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<SrvRequest*> pending;
  std::unordered_map<uint64_t, SrvRequest*> requests;
  std::vector<SrvBatch*> inflight;
  uint64_t next_ticket = 1;
  int inflight_requests = 0;
  double sms_in_use = 0;
  bool stop = false;
  std::thread worker;
  // statistics
  std::vector<double> latencies;
  int64_t submitted = 0, completed = 0, failed = 0, options = 0, batches = 0;
  double t_first = 0, t_last = 0;
};

namespace {

void server_retire(lvc_server* S) {
  for (auto it = S->inflight.begin(); it != S->inflight.end();) {
    SrvBatch* b = *it;
    const cudaError_t q = cudaEventQuery(b->done);
    if (q == cudaErrorNotReady) {
      ++it;
      continue;
    }
    const double t = now_s();
    double* host = S->pinned[b->stream];
    const int64_t np = b->plan->nprices;
    const int derr = q == cudaSuccess ? reinterpret_cast<const int*>(host + np)[0] : 1;
    int64_t off = 0;
    for (SrvRequest* r : b->reqs) {
      r->t_done = t;
      if (q != cudaSuccess || derr) {
        r->status = 2;
        r->error = q != cudaSuccess ? std::string("CUDA error: ") + cudaGetErrorString(q)
                                    : "rollback kernel rejected a work item";
        S->failed++;
      } else {
        r->prices.assign(host + off, host + off + r->c.outer);
        r->status = 1;
        S->completed++;
        S->options += r->c.outer;
        S->latencies.push_back(t - r->t_submit);
        S->t_last = t;
      }
      off += r->c.outer;
    }
    S->inflight_requests -= (int)b->reqs.size();
    S->sms_in_use -= b->sms;
    if (S->sms_in_use < 1e-9) S->sms_in_use = 0;
    S->stream_busy[b->stream] = false;
    cudaEventDestroy(b->done);
    if (b->cached && q == cudaSuccess && !derr) {
      const lvc_calibration& c = b->reqs[0]->c;
      auto key = std::make_tuple((int)c.outer, (int)c.numX, (int)c.numY, (int)c.numT);
      S->plan_cache[key].push_back(b->plan);
      S->plan_lru.push_back({key, b->plan});
    } else {
      plan_release(b->plan);
    }
    // a batch completed: grow a backed-off batch size again toward the configured one
    if (q == cudaSuccess && S->cfg.max_batch_requests < S->max_batch_configured)
      S->cfg.max_batch_requests = std::min(S->max_batch_configured, 2 * S->cfg.max_batch_requests);
    delete b;
    it = S->inflight.erase(it);
  }
}

// Device bytes a one-calibration plan takes (tables, pivots, work list,
// prices, state scratch), from the same layouts the plan builder uses.
size_t request_bytes(const futhark_context* ctx, const lvc_calibration& c, int precision) {
  const bool f64 = precision == LVC_F64;
  const Config cf = f64 ? choose_config<double>(ctx, c.numX, c.numY)
                        : choose_config<float>(ctx, c.numX, c.numY);
  const int Xp = std::max(8, pow2ceil(c.numX));
  const size_t ps = f64 ? 8 : 4;
  size_t b = 8 * (size_t)al2(tab_layout(c.numX, c.numY, c.numT, Xp, cf.kind).total);
  b += ps * (size_t)(piv_elems(c.numX, c.numY, c.numT, Xp, cf.kind, cf.ld) + 4);
  b += 16 * (size_t)c.outer + 4096;
  if (cf.gstate) b += ps * (size_t)cf.grid_elems * 148 * 4;
  return b + 8 * 256;  // allocation rounding
}

// Admits one batch from the front of the queue; returns false when nothing
// could be admitted.  Called with S->mu held; releases it while building.
bool server_admit(lvc_server* S, std::unique_lock<std::mutex>& lk) {
  if (S->pending.empty()) return false;
  if (std::find(S->stream_busy.begin(), S->stream_busy.end(), false) == S->stream_busy.end()) return false;
  // Admission order: shortest job first (option-cell-steps), so that small
  // requests are not queued behind large ones; a request that has waited
  // longer than kStarveS goes first (oldest first), so large ones are not
  // starved.
  constexpr double kStarveS = 0.05;
  constexpr double kBatchSpread = 4.0;     // largest / first request of a batch, by work
  constexpr double kSmallBatchWork = 1.5e8;  // option-cell-steps (about a millisecond of the GPU)
  const double tnow = now_s();
  auto next_pick = [&]() {
    auto best = S->pending.end();
    for (auto it = S->pending.begin(); it != S->pending.end(); ++it) {
      if (tnow - (*it)->t_submit > kStarveS) return it;  // the deque is in arrival order
      if (best == S->pending.end() || (*it)->work < (*best)->work) best = it;
    }
    return best;
  };
  std::vector<SrvRequest*> take;
  size_t bytes = 0;
  auto free_bytes = [&]() { return S->pool.budget > S->pool.in_use ? S->pool.budget - S->pool.in_use : 0; };
  double take_work = 0, first_work = 0;
  while (!S->pending.empty() && (int)take.size() < S->cfg.max_batch_requests &&
         S->inflight_requests + (int)take.size() < S->cfg.max_inflight_requests) {
    auto pit = next_pick();
    SrvRequest* r = *pit;
    // a batch completes with its largest request: a small request joins no
    // batch of requests much larger than itself
    if (!take.empty() && r->work > kBatchSpread * first_work) break;
    const size_t rb = request_bytes(&S->sctx, r->c, S->cfg.precision);
    if (rb > S->pool.budget) {  // can never fit: fail it now
      S->pending.erase(pit);
      r->status = 2;
      r->error = "request needs more device memory than the server's HBM budget";
      r->t_done = now_s();
      S->failed++;
      S->cv_done.notify_all();
      continue;
    }
    // idle cached plans give their memory back before a request is refused
    while (bytes + rb > free_bytes() && !S->plan_lru.empty()) {
      auto victim = S->plan_lru.front();
      S->plan_lru.pop_front();
      auto& v = S->plan_cache[victim.first];
      v.erase(std::find(v.begin(), v.end(), victim.second));
      plan_release(victim.second);
    }
    if (bytes + rb > free_bytes()) break;
    if (take.empty()) first_work = r->work;
    take.push_back(r);
    take_work += r->work;
    bytes += rb;
    S->pending.erase(pit);
  }
  if (take.empty()) return false;
  // a free stream: a small batch prefers the high-priority ones, a large one
  // the others (either takes what is free)
  const bool small = take_work <= kSmallBatchWork;
  int si = -1;
  for (int pass = 0; pass < 2 && si < 0; pass++)
    for (size_t i = 0; i < S->streams.size(); i++)
      if (!S->stream_busy[i] && (pass == 1 || S->stream_high[i] == small)) {
        si = (int)i;
        break;
      }
  std::vector<lvc_calibration> cs;
  for (SrvRequest* r : take) cs.push_back(r->c);
  S->stream_busy[si] = true;
  // a one-request batch reuses an idle plan of the same sizes when there is one
  lvc_plan* P = nullptr;
  if (take.size() == 1) {
    const lvc_calibration& c = take[0]->c;
    auto key = std::make_tuple((int)c.outer, (int)c.numX, (int)c.numY, (int)c.numT);
    auto ci = S->plan_cache.find(key);
    if (ci != S->plan_cache.end() && !ci->second.empty()) {
      P = ci->second.back();
      ci->second.pop_back();
      for (auto li = S->plan_lru.begin(); li != S->plan_lru.end(); ++li)
        if (li->second == P) {
          S->plan_lru.erase(li);
          break;
        }
      S->plans_reused++;
    }
  }
  const bool reused = P != nullptr;
  lk.unlock();
  int rc = 0;
  cudaError_t e = cudaSuccess;
  cudaStream_t st = S->streams[si];
  if (reused) {
    // new scalars into the plan's calibration record, uploaded on the batch's stream
    fill_scalars(P->calibs[0], cs[0]);
    P->params[0] = cs[0];
    e = cudaMemcpyAsync(P->d_calibs, P->calibs.data(), sizeof(CalibDev), cudaMemcpyHostToDevice, st);
  } else {
    rc = plan_new_locked(&S->sctx, cs.data(), (int)cs.size(), S->cfg.precision, &P, &S->pool,
                         /*use_graph=*/false, /*max_sms=*/-1);
  }
  SrvBatch* b = nullptr;
  if (!rc && e == cudaSuccess) {
    b = new SrvBatch();
    b->reqs = take;
    b->plan = P;
    b->cached = take.size() == 1;
    b->stream = si;
    b->sms = P->sms;
    b->t_launch = now_s();
    if (S->pinned_cap[si] < P->nprices + 1) {
      // outgrown staging is kept until the server is freed: cudaFreeHost
      // would synchronise the device under the running batches
      if (S->pinned[si]) S->pinned_retired.push_back(S->pinned[si]);
      S->pinned[si] = nullptr;
      S->pinned_cap[si] = std::max<int64_t>(2 * (P->nprices + 1), 1 << 16);
      e = cudaMallocHost((void**)&S->pinned[si], sizeof(double) * S->pinned_cap[si]);
      if (e != cudaSuccess) S->pinned_cap[si] = 0;
    }
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming);
    if (e == cudaSuccess) e = plan_enqueue(P, st, nullptr);
    if (e == cudaSuccess && P->nprices > 0)
      e = cudaMemcpyAsync(S->pinned[si], P->d_out, sizeof(double) * P->nprices, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) {
      // the kernels' error flag, in the slot after the prices
      int* flag = reinterpret_cast<int*>(S->pinned[si] + P->nprices);
      e = cudaMemcpyAsync(flag, P->d_err, sizeof(int), cudaMemcpyDeviceToHost, st);
    }
    if (e == cudaSuccess) e = cudaEventRecord(b->done, st);
  }
  lk.lock();
  if (rc == FUTHARK_OUT_OF_MEMORY && (!S->inflight.empty() || take.size() > 1)) {
    // the budget is taken by running batches (or fragmented): retry with
    // fewer requests, or when running batches complete
    if (P) plan_release(P);
    // the taken requests go back in arrival order
    auto requeue = [&]() {
      for (SrvRequest* r : take) {
        auto at = std::find_if(S->pending.begin(), S->pending.end(),
                               [&](const SrvRequest* q) { return q->t_submit > r->t_submit; });
        S->pending.insert(at, r);
      }
    };
    requeue();
    S->stream_busy[si] = false;
    if (S->inflight.empty()) {
      // back off to half the batch; completed batches restore it (server_retire)
      S->cfg.max_batch_requests = std::max<int32_t>(1, (int32_t)take.size() / 2);
      return true;  // try again at once with the smaller batch size
    }
    return false;
  }
  if (rc || e != cudaSuccess) {
    const std::string msg = rc ? S->sctx.error : std::string("CUDA error: ") + cudaGetErrorString(e);
    for (SrvRequest* r : take) {
      r->status = 2;
      r->error = msg;
      r->t_done = now_s();
      S->failed++;
    }
    if (b) {
      if (b->done) cudaEventDestroy(b->done);
      plan_release(b->plan);
      delete b;
    } else if (P) {
      plan_release(P);
    }
    S->stream_busy[si] = false;
    S->cv_done.notify_all();
    return true;
  }
  S->inflight.push_back(b);
  S->inflight_requests += (int)take.size();
  S->sms_in_use += b->sms;
  S->batches++;
  return true;
}

void server_loop(lvc_server* S) {
  cudaSetDevice(S->sctx.device);
  std::unique_lock<std::mutex> lk(S->mu);
  while (true) {
    const size_t before = S->inflight.size();
    server_retire(S);
    if (S->inflight.size() != before) S->cv_done.notify_all();
    while (server_admit(S, lk)) {
    }
    if (S->stop && S->pending.empty() && S->inflight.empty()) break;
    if (S->inflight.empty()) {
      S->cv_work.wait(lk, [&] { return S->stop || !S->pending.empty(); });
    } else {
      S->cv_work.wait_for(lk, std::chrono::microseconds(20));
    }
  }
}

}  // namespace

extern "C" {

int lvc_server_new(struct futhark_context* ctx, const struct lvc_server_config* cfg,
                   struct lvc_server** out) {
  std::lock_guard<std::mutex> g(ctx->mu);
  if (!ctx->ok) return set_error(ctx, FUTHARK_PROGRAM_ERROR, "context has no usable CUDA device");
  lvc_server_config c = cfg ? *cfg : lvc_server_config{};
  if (c.precision != LVC_F64 && c.precision != LVC_F32_STATE)
    return set_error(ctx, FUTHARK_PROGRAM_ERROR, "unknown precision");
  if (c.max_inflight_requests <= 0) c.max_inflight_requests = 256;
  if (c.max_batch_requests <= 0) c.max_batch_requests = 64;
  if (c.num_streams <= 0) c.num_streams = 8;
  if (c.hbm_budget_bytes <= 0) c.hbm_budget_bytes = int64_t(8) << 30;
  LVC_CUDA(ctx, cudaSetDevice(ctx->device));
  lvc_server* S = new lvc_server();
  S->user_ctx = ctx;
  S->cfg = c;
  S->max_batch_configured = c.max_batch_requests;
  S->sctx.device = ctx->device;
  S->sctx.num_sms = ctx->num_sms;
  S->sctx.max_smem = ctx->max_smem;
  S->sctx.shapes = ctx->shapes;  // the server prices with the shapes tuned so far (ctx->mu is held)
  S->sctx.tuning = ctx->tuning;
  S->sctx.ok = true;
  S->pool.budget = (size_t)c.hbm_budget_bytes;
  cudaError_t e = cudaStreamCreateWithFlags(&S->sctx.stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&S->sctx.capture, cudaStreamNonBlocking);
  // half the streams at the device's greatest priority: the block scheduler
  // starts their CTAs ahead of waiting CTAs of the other half's large batches
  int prio_low = 0, prio_high = 0;
  if (cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high) != cudaSuccess) prio_low = prio_high = 0;
  for (int i = 0; i < c.num_streams && e == cudaSuccess; i++) {
    cudaStream_t st;
    const bool high = 2 * i < c.num_streams;
    e = cudaStreamCreateWithPriority(&st, cudaStreamNonBlocking, high ? prio_high : prio_low);
    if (e == cudaSuccess) {
      S->streams.push_back(st);
      S->stream_busy.push_back(false);
      S->stream_high.push_back(high);
      // staging for 65535 prices and the error flag; a larger batch grows it
      double* pin = nullptr;
      e = cudaMallocHost((void**)&pin, sizeof(double) << 16);
      S->pinned.push_back(e == cudaSuccess ? pin : nullptr);
      S->pinned_cap.push_back(e == cudaSuccess ? (1 << 16) : 0);
    }
  }
  // reserve the whole budget up front: serving never reaches cudaMalloc
  if (e == cudaSuccess) {
    char* blk = S->pool.grow((size_t)c.hbm_budget_bytes);
    if (blk) S->pool.insert_free(blk, (size_t)c.hbm_budget_bytes); else e = cudaErrorMemoryAllocation;
  }
  if (e != cudaSuccess) {
    for (cudaStream_t st : S->streams) cudaStreamDestroy(st);
    for (double* pin : S->pinned)
      if (pin) cudaFreeHost(pin);
    if (S->sctx.stream) cudaStreamDestroy(S->sctx.stream);
    if (S->sctx.capture) cudaStreamDestroy(S->sctx.capture);
    delete S;
    return cuda_fail(ctx, e, "lvc_server_new");
  }
  S->worker = std::thread(server_loop, S);
  *out = S;
  return 0;
}

int lvc_server_submit(struct lvc_server* S, const struct lvc_calibration* c, uint64_t* ticket) {
  {
    std::lock_guard<std::mutex> g(S->user_ctx->mu);
    if (int rc = validate(S->user_ctx, *c, 0)) return rc;
  }
  SrvRequest* r = new SrvRequest();
  r->c = *c;
  r->work = (double)c->outer * c->numX * c->numY * (c->numT > 1 ? c->numT - 1 : 0);
  r->t_submit = now_s();
  {
    std::lock_guard<std::mutex> g(S->mu);
    r->ticket = S->next_ticket++;
    S->requests[r->ticket] = r;
    S->pending.push_back(r);
    S->submitted++;
    if (S->t_first == 0) S->t_first = r->t_submit;
  }
  S->cv_work.notify_one();
  *ticket = r->ticket;
  return 0;
}

int lvc_server_poll(struct lvc_server* S, uint64_t ticket, int32_t* done) {
  std::lock_guard<std::mutex> g(S->mu);
  auto it = S->requests.find(ticket);
  if (it == S->requests.end()) return FUTHARK_PROGRAM_ERROR;
  *done = it->second->status != 0;
  return 0;
}

int lvc_server_wait(struct lvc_server* S, uint64_t ticket, double* prices, double timeout_s) {
  std::unique_lock<std::mutex> lk(S->mu);
  auto it = S->requests.find(ticket);
  if (it == S->requests.end()) {
    std::lock_guard<std::mutex> g(S->user_ctx->mu);
    return set_error(S->user_ctx, FUTHARK_PROGRAM_ERROR, "unknown ticket");
  }
  SrvRequest* r = it->second;
  const auto deadline = std::chrono::steady_clock::now() +
                        std::chrono::duration<double>(timeout_s > 0 ? timeout_s : 1e9);
  if (!S->cv_done.wait_until(lk, deadline, [&] { return r->status != 0; })) {
    std::lock_guard<std::mutex> g(S->user_ctx->mu);
    return set_error(S->user_ctx, FUTHARK_PROGRAM_ERROR, "timed out waiting for the request");
  }
  S->requests.erase(it);
  const int status = r->status;
  const std::string err = r->error;
  if (status == 1 && prices && !r->prices.empty())
    memcpy(prices, r->prices.data(), sizeof(double) * r->prices.size());
  delete r;
  lk.unlock();
  if (status != 1) {
    std::lock_guard<std::mutex> g(S->user_ctx->mu);
    return set_error(S->user_ctx, FUTHARK_PROGRAM_ERROR, err);
  }
  return 0;
}

int lvc_server_stats(struct lvc_server* S, struct lvc_server_stats* st) {
  std::lock_guard<std::mutex> g(S->mu);
  memset(st, 0, sizeof *st);
  st->submitted = S->submitted;
  st->completed = S->completed;
  st->failed = S->failed;
  st->options = S->options;
  st->batches = S->batches;
  st->span_s = S->t_last > S->t_first ? S->t_last - S->t_first : 0.0;
  st->throughput_options_per_s = st->span_s > 0 ? S->options / st->span_s : 0.0;
  if (!S->latencies.empty()) {
    std::vector<double> v = S->latencies;
    std::sort(v.begin(), v.end());
    auto pct = [&](double p) { return 1e3 * v[std::min(v.size() - 1, (size_t)(p * (v.size() - 1) + 0.5))]; };
    st->p50_ms = pct(0.50);
    st->p99_ms = pct(0.99);
    st->max_ms = 1e3 * v.back();
    double sum = 0;
    for (double x : v) sum += x;
    st->mean_ms = 1e3 * sum / v.size();
  }
  st->hbm_reserved_bytes = (int64_t)S->pool.reserved;
  return 0;
}

int lvc_server_reset_stats(struct lvc_server* S) {
  std::lock_guard<std::mutex> g(S->mu);
  S->latencies.clear();
  S->submitted = S->completed = S->failed = S->options = S->batches = 0;
  S->t_first = S->t_last = 0;
  return 0;
}

int lvc_server_free(struct lvc_server* S) {
  if (!S) return 0;
  {
    std::lock_guard<std::mutex> g(S->mu);
    S->stop = true;
  }
  S->cv_work.notify_all();
  if (S->worker.joinable()) S->worker.join();
  cudaSetDevice(S->sctx.device);
  for (auto& kv : S->requests) delete kv.second;
  for (size_t i = 0; i < S->streams.size(); i++) {
    cudaStreamSynchronize(S->streams[i]);
    cudaStreamDestroy(S->streams[i]);
    if (S->pinned[i]) cudaFreeHost(S->pinned[i]);
  }
  for (double* p : S->pinned_retired) cudaFreeHost(p);
  for (auto& kv : S->plan_cache)
    for (lvc_plan* P : kv.second) plan_release(P);
  cudaStreamDestroy(S->sctx.stream);
  cudaStreamDestroy(S->sctx.capture);
  delete S;
  return 0;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Batched tridiagonal solvers: the entry points of the tridiagonal test
// program (misc/ocean-sim/tridiag-test.fut:14-26) on the same contexts.
// ---------------------------------------------------------------------------
namespace {

constexpr int64_t kTridagInnerDim = 115;  // INNER_DIM of tridiag-test.fut:4

// Synchronises ctx->stream and reports a bounded device wait that gave up.
// Called with ctx->mu held.
int tridag_check_locked(futhark_context* ctx) {
  int flag = 0;  // a bounded device wait that gave up
  LVC_CUDA(ctx, cudaMemcpyFromSymbolAsync(&flag, lvc_tridag_err, sizeof flag, 0, cudaMemcpyDeviceToHost, ctx->stream));
  LVC_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (flag) {
    const int zero = 0;
    cudaMemcpyToSymbol(lvc_tridag_err, &zero, sizeof zero);
    return set_error(ctx, FUTHARK_PROGRAM_ERROR, "tridiagonal solve: a bounded device wait timed out");
  }
  return 0;
}

// Enqueues one batched solve on ctx->stream (device pointers).  Called with
// ctx->mu held.  m <= 256: the tensor-memory kernel; m <= 400: the
// streaming kernel, no scratch; larger m: scratch from the context's device
// pool (stream-ordered: every user of that pool runs on ctx->stream).
// cuTensorMapEncodeTiled from the driver, looked up once through the runtime
// (the library does not link against the driver library itself); null where
// the driver does not offer it.
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

// The [rows / 4][4m] group view of one input of a batch with odd m and
// rows % 4 == 0, in boxes of kTriTmaGroups groups x kTriTmaBox floats
// (lvc_tridag_tma_kernel); false where it cannot be made (no encoder, a base
// address off the 16-byte grid the tensor copies need).
bool tri_group_map(CUtensorMap* map, const float* p, int64_t rows, int64_t m) {
  const PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
  if (!enc || (reinterpret_cast<uintptr_t>(p) & 15u) != 0) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)(4 * m), (cuuint64_t)(rows / 4)};
  const cuuint64_t strides[1] = {(cuuint64_t)(4 * m) * sizeof(float)};
  const cuuint32_t box[2] = {(cuuint32_t)kTriTmaBox, (cuuint32_t)kTriTmaGroups};
  const cuuint32_t estr[2] = {1, 1};
  return enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(p), dims, strides, box, estr,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Raises a tridiagonal kernel's dynamic shared-memory limit once per context
// (each kernel instance always asks for the same size).
int tri_smem_limit(futhark_context* ctx, const void* fn, size_t bytes) {
  if (ctx->tri_smem_raised.count(fn)) return 0;
  LVC_CUDA(ctx, cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  ctx->tri_smem_raised.insert(fn);
  return 0;
}

int tridag_launch(futhark_context* ctx, int form, int64_t rows, int64_t m, const float* a, const float* b,
                  const float* c, const float* y, float* out) {
  if (rows < 0 || m < 0 || m > INT32_MAX) return set_error(ctx, FUTHARK_PROGRAM_ERROR, "bad tridiagonal batch shape");
  if (rows == 0 || m == 0) return 0;
  if (m <= kTriTmemMaxM && (m & 1) && rows % 4 == 0 && rows / 4 <= INT32_MAX - kTriTmaGroups) {
    // odd m: inputs staged for the whole CTA by tensor copies of 4-system groups
    const float* src[4] = {a, b, c, y};
    bool ok = ctx->tri_map_rows == rows && ctx->tri_map_m == m;
    for (int i = 0; i < 4 && ok; i++) ok = ctx->tri_map_src[i] == src[i];
    if (!ok) {  // encode the maps of this batch (host work: reused while the batch repeats)
      ok = true;
      for (int i = 0; i < 4 && ok; i++) ok = tri_group_map(&ctx->tri_maps[i], src[i], rows, m);
      ctx->tri_map_rows = ok ? rows : -1;
      ctx->tri_map_m = ok ? m : -1;
      for (int i = 0; i < 4; i++) ctx->tri_map_src[i] = ok ? src[i] : nullptr;
    }
    if (ok) {
      const CUtensorMap* maps = ctx->tri_maps;
      const int64_t nblk = (rows + 32 * kTriTmemWarps - 1) / (32 * kTriTmemWarps);
      const int cols = tri_tmem_cols((int)m);
      auto fk = cols == 256 ? (form == 0 ? lvc_tridag_tma_kernel<0, 256> : lvc_tridag_tma_kernel<1, 256>)
                            : (form == 0 ? lvc_tridag_tma_kernel<0, 512> : lvc_tridag_tma_kernel<1, 512>);
      const size_t smem = tri_tma_smem(cols);
      if (int rc = tri_smem_limit(ctx, (const void*)fk, smem)) return rc;
      fk<<<(unsigned)nblk, kTriTmaThreads, smem, ctx->stream>>>(maps[0], maps[1], maps[2], maps[3], rows,
                                                                     (int)m, out);
      const cudaError_t e = cudaGetLastError();
      if (e != cudaSuccess) return cuda_fail(ctx, e, "tridiagonal launch");
      return 0;
    }
  }
  if (m <= kTriTmemMaxM) {  // intermediates in tensor memory, four warps per CTA
    const int64_t nblk = (rows + 32 * kTriTmemWarps - 1) / (32 * kTriTmemWarps);
    if (nblk > INT32_MAX) return set_error(ctx, FUTHARK_PROGRAM_ERROR, "tridiagonal batch too large");
    const int cols = tri_tmem_cols((int)m);
    auto fk = cols == 256 ? (form == 0 ? lvc_tridag_tmem_kernel<0, 256> : lvc_tridag_tmem_kernel<1, 256>)
                          : (form == 0 ? lvc_tridag_tmem_kernel<0, 512> : lvc_tridag_tmem_kernel<1, 512>);
    const size_t smem = tri_tmem_smem(cols);
    if (int rc = tri_smem_limit(ctx, (const void*)fk, smem)) return rc;
    fk<<<(unsigned)nblk, 32 * kTriTmemWarps, smem, ctx->stream>>>(rows, (int)m, a, b, c, y, out);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(ctx, e, "tridiagonal launch");
    return 0;
  }
  if (m <= kTriMaxM) {  // inputs streamed, intermediates in shared memory
    const int64_t nblk = (rows + 31) / 32;
    if (nblk > INT32_MAX) return set_error(ctx, FUTHARK_PROGRAM_ERROR, "tridiagonal batch too large");
    const size_t smem = sizeof(float) * (size_t)tri_stream_floats((int)m);
    const size_t smem_max = sizeof(float) * (size_t)tri_stream_floats(kTriMaxM);
    auto fs = form == 0 ? lvc_tridag_stream_kernel<0> : lvc_tridag_stream_kernel<1>;
    if (int rc = tri_smem_limit(ctx, (const void*)fs, smem_max)) return rc;
    fs<<<(unsigned)nblk, 32, smem, ctx->stream>>>(rows, (int)m, a, b, c, y, out);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(ctx, e, "tridiagonal launch");
    return 0;
  }
  const int64_t blocks = (rows + kTriThreads - 1) / kTriThreads;
  if (blocks > INT32_MAX) return set_error(ctx, FUTHARK_PROGRAM_ERROR, "tridiagonal batch too large");
  if (!ctx->pool) ctx->pool = new DevicePool();
  float* gscratch = static_cast<float*>(ctx->pool->alloc(sizeof(float) * (size_t)m * (size_t)rows));
  if (!gscratch) return set_error(ctx, FUTHARK_OUT_OF_MEMORY, "out of device memory for tridiagonal scratch");
  auto fn = form == 0 ? lvc_tridag_kernel<0> : lvc_tridag_kernel<1>;
  fn<<<(unsigned)blocks, kTriThreads, 0, ctx->stream>>>(rows, (int)m, a, b, c, y, out, gscratch);
  const cudaError_t e = cudaGetLastError();
  ctx->pool->release(gscratch);  // later users of the pool are ordered after this launch
  if (e != cudaSuccess) return cuda_fail(ctx, e, "tridiagonal launch");
  return 0;
}

int tridag_entry(futhark_context* ctx, futhark_f32_2d** out0, const futhark_f32_2d* a, const futhark_f32_2d* b,
                 const futhark_f32_2d* c, const futhark_f32_2d* y, int form, int64_t need_m) {
  std::lock_guard<std::mutex> g(ctx->mu);
  if (!ctx->ok) return set_error(ctx, FUTHARK_PROGRAM_ERROR, "context has no usable CUDA device");
  if (!out0 || !a || !b || !c || !y) return set_error(ctx, FUTHARK_PROGRAM_ERROR, "null array");
  const int64_t rows = a->shape[0], m = a->shape[1];
  for (const futhark_f32_2d* v : {b, c, y})
    if (v->shape[0] != rows || v->shape[1] != m)
      return set_error(ctx, FUTHARK_PROGRAM_ERROR, "tridiagonal entry: the four input arrays differ in shape");
  if (need_m >= 0 && m != need_m) {
    char buf[160];
    snprintf(buf, sizeof buf, "tridiagonal entry: inner dimension %lld does not match the required %lld",
             (long long)m, (long long)need_m);
    return set_error(ctx, FUTHARK_PROGRAM_ERROR, buf);
  }
  LVC_CUDA(ctx, cudaSetDevice(ctx->device));
  auto* o = new (std::nothrow) futhark_f32_2d();
  if (!o) return set_error(ctx, FUTHARK_OUT_OF_MEMORY, "out of host memory");
  o->shape[0] = rows;
  o->shape[1] = m;
  o->bytes = sizeof(float) * (size_t)std::max<int64_t>(1, rows * m);
  if (!(o->data = static_cast<float*>(arr_alloc(ctx, o->bytes)))) {
    delete o;
    return set_error(ctx, FUTHARK_OUT_OF_MEMORY, "out of device memory");
  }
  int rc = tridag_launch(ctx, form, rows, m, a->data, b->data, c->data, y->data, o->data);
  if (!rc) rc = tridag_check_locked(ctx);
  if (rc) {
    arr_free(ctx, o->data);
    delete o;
    return rc;
  }
  *out0 = o;
  return 0;
}

}  // namespace

extern "C" {

struct futhark_f32_2d* futhark_new_f32_2d(struct futhark_context* ctx, const float* data, int64_t dim0,
                                          int64_t dim1) {
  std::lock_guard<std::mutex> g(ctx->mu);
  if (!ctx->ok || dim0 < 0 || dim1 < 0) {
    ctx->error = "cannot create array";
    return nullptr;
  }
  cudaSetDevice(ctx->device);
  auto* a = new (std::nothrow) futhark_f32_2d();
  if (!a) return nullptr;
  a->shape[0] = dim0;
  a->shape[1] = dim1;
  const int64_t n = dim0 * dim1;
  a->bytes = sizeof(float) * (size_t)std::max<int64_t>(1, n);
  if (!(a->data = static_cast<float*>(arr_alloc(ctx, a->bytes)))) {
    ctx->error = "out of device memory";
    delete a;
    return nullptr;
  }
  if (n > 0 && data &&
      cudaMemcpyAsync(a->data, data, sizeof(float) * n, cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess) {
    arr_free(ctx, a->data);
    delete a;
    ctx->error = "host to device copy failed";
    return nullptr;
  }
  cudaStreamSynchronize(ctx->stream);
  return a;
}

int futhark_free_f32_2d(struct futhark_context* ctx, struct futhark_f32_2d* arr) {
  if (!arr) return 0;
  std::lock_guard<std::mutex> g(ctx->mu);
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  arr_free(ctx, arr->data);
  delete arr;
  return 0;
}

int futhark_values_f32_2d(struct futhark_context* ctx, struct futhark_f32_2d* arr, float* data) {
  std::lock_guard<std::mutex> g(ctx->mu);
  if (!arr) return set_error(ctx, FUTHARK_PROGRAM_ERROR, "null array");
  LVC_CUDA(ctx, cudaSetDevice(ctx->device));
  const int64_t n = arr->shape[0] * arr->shape[1];
  if (n > 0)
    LVC_CUDA(ctx, cudaMemcpyAsync(data, arr->data, sizeof(float) * n, cudaMemcpyDeviceToHost, ctx->stream));
  LVC_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return 0;
}

const int64_t* futhark_shape_f32_2d(struct futhark_context* ctx, struct futhark_f32_2d* arr) {
  (void)ctx;
  return arr ? arr->shape : nullptr;
}

int futhark_entry_tridagNested(struct futhark_context* ctx, struct futhark_f32_2d** out0,
                               const struct futhark_f32_2d* in0, const struct futhark_f32_2d* in1,
                               const struct futhark_f32_2d* in2, const struct futhark_f32_2d* in3) {
  return tridag_entry(ctx, out0, in0, in1, in2, in3, 1, -1);
}
int futhark_entry_tridagNestedConst(struct futhark_context* ctx, struct futhark_f32_2d** out0,
                                    const struct futhark_f32_2d* in0, const struct futhark_f32_2d* in1,
                                    const struct futhark_f32_2d* in2, const struct futhark_f32_2d* in3) {
  return tridag_entry(ctx, out0, in0, in1, in2, in3, 1, kTridagInnerDim);
}
int futhark_entry_tridagNestedSeq(struct futhark_context* ctx, struct futhark_f32_2d** out0,
                                  const struct futhark_f32_2d* in0, const struct futhark_f32_2d* in1,
                                  const struct futhark_f32_2d* in2, const struct futhark_f32_2d* in3) {
  return tridag_entry(ctx, out0, in0, in1, in2, in3, 0, -1);
}
int futhark_entry_tridagNestedSeqConst(struct futhark_context* ctx, struct futhark_f32_2d** out0,
                                       const struct futhark_f32_2d* in0, const struct futhark_f32_2d* in1,
                                       const struct futhark_f32_2d* in2, const struct futhark_f32_2d* in3) {
  return tridag_entry(ctx, out0, in0, in1, in2, in3, 0, kTridagInnerDim);
}

int lvc_tridag_f32(struct futhark_context* ctx, int32_t form, int64_t rows, int64_t m, const float* a,
                   const float* b, const float* c, const float* y, float* out) {
  std::lock_guard<std::mutex> g(ctx->mu);
  if (!ctx->ok) return set_error(ctx, FUTHARK_PROGRAM_ERROR, "context has no usable CUDA device");
  if (form != LVC_TRIDAG_SEQ && form != LVC_TRIDAG_PAR)
    return set_error(ctx, FUTHARK_PROGRAM_ERROR, "unknown tridiagonal form");
  if (rows * m > 0 && (!a || !b || !c || !y || !out)) return set_error(ctx, FUTHARK_PROGRAM_ERROR, "null pointer");
  LVC_CUDA(ctx, cudaSetDevice(ctx->device));
  return tridag_launch(ctx, form == LVC_TRIDAG_SEQ ? 0 : 1, rows, m, a, b, c, y, out);
}

int lvc_tridag_check(struct futhark_context* ctx) {
  std::lock_guard<std::mutex> g(ctx->mu);
  if (!ctx->ok) return set_error(ctx, FUTHARK_PROGRAM_ERROR, "context has no usable CUDA device");
  LVC_CUDA(ctx, cudaSetDevice(ctx->device));
  return tridag_check_locked(ctx);
}

int lvc_wait_selftest(struct futhark_context* ctx, int32_t polls, int32_t arrive) {
  std::lock_guard<std::mutex> g(ctx->mu);
  if (!ctx->ok) return set_error(ctx, FUTHARK_PROGRAM_ERROR, "context has no usable CUDA device");
  if (polls < 1 || polls > kWaitPolls) return set_error(ctx, FUTHARK_PROGRAM_ERROR, "polls out of range");
  LVC_CUDA(ctx, cudaSetDevice(ctx->device));
  lvc_wait_selftest_kernel<<<1, 32, 0, ctx->stream>>>(polls, arrive);
  LVC_CUDA(ctx, cudaGetLastError());
  return tridag_check_locked(ctx);
}

}  // extern "C"
