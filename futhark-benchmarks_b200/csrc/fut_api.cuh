// The context, configuration and array plumbing of the C API the Futhark
// compiler generates for a program, shared by the engine's one-program
// libraries (libtke.so, libop.so).  Include it exactly once per library,
// after the library's public header (which declares the exported functions
// with default visibility).  It defines futhark_context_config,
// futhark_context, the array types futhark_f32_1d/2d/3d and futhark_i32_1d/2d
// (device storage shared between arrays by reference count, so an entry
// point can return an input unchanged without a copy), the context functions,
// and FUT_ARRAY_API, which a library expands for the array types its entry
// points use.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <string>

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
  void* scratch = nullptr;  // the entry point's scratch, grown on demand
  size_t scratch_bytes = 0;
  int reduce_order = 0;        // OptionPricing: 0 f64 accumulation, 1 the reference's f32 running sum
  cudaStream_t aux = nullptr;  // a second stream for work that overlaps `stream`'s,
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;  // forked and joined by these events
  bool smem_raised = false;    // a kernel's shared-memory limit already raised on this device
};

namespace {

// Device storage shared by the arrays that view it, so that an entry point can
// return a consumed input unchanged as an output without copying it.
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
struct futhark_i32_1d : DevArray<int32_t, 1> {};
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

// Creates the context's auxiliary stream and its fork/join events on first
// use (lock held, device set).
bool ensure_aux_stream(futhark_context* ctx) {
  if (ctx->aux) return true;
  if (cudaStreamCreateWithFlags(&ctx->aux, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&ctx->ev_join, cudaEventDisableTiming) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return true;
}

// Grows the context's scratch to at least `bytes` (lock held, device set).
bool ensure_scratch(futhark_context* ctx, size_t bytes) {
  if (ctx->scratch_bytes >= bytes) return true;
  cudaStreamSynchronize(ctx->stream);
  if (ctx->scratch) cudaFree(ctx->scratch);
  ctx->scratch = nullptr;
  ctx->scratch_bytes = 0;
  if (cudaMalloc(&ctx->scratch, bytes) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  ctx->scratch_bytes = bytes;
  return true;
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
    if (ctx->aux) {
      cudaStreamSynchronize(ctx->aux);
      cudaStreamDestroy(ctx->aux);
      cudaEventDestroy(ctx->ev_fork);
      cudaEventDestroy(ctx->ev_join);
    }
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

#define FUT_ARRAY_API(NAME, T, R, ...)                                                                 \
  struct futhark_##NAME* futhark_new_##NAME(struct futhark_context* ctx, const T* data, __VA_ARGS__) { \
    const int64_t dims[] = {FUT_DIMS_##R};                                                             \
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
#define FUT_DIMS_1 dim0
#define FUT_DIMS_2 dim0, dim1
#define FUT_DIMS_3 dim0, dim1, dim2

}  // extern "C"
