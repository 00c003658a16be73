/*
 * LocVolCalib.h -- C API of the B200 LocVolCalib engine (liblvc.so).
 *
 * Part 1 is the header that `futhark cuda --library finpar/LocVolCalib.fut`
 * would generate for the reference program: the same context/config life
 * cycle, the same `futhark_entry_main` signature (outputs first, then the nine
 * scalar inputs of `main`, finpar/LocVolCalib.fut:238-246) and the same array
 * accessors.  A C host written against the generated library links against
 * liblvc.so instead, unchanged.  The shape of that API is witnessed in the
 * reference by its in-repo consumer, the lys front-end (cited per function).
 *
 * Part 2 adds the f64 twin of the entry point and the engine's batched and
 * serving forms, which have no counterpart in the generated API.
 *
 * Conventions (as in the generated API): functions returning int return 0 on
 * success and a non-zero error code on failure, with a message available from
 * futhark_context_get_error.  Invalid sizes are reported as errors, never by
 * aborting the process.
 */
#ifndef LOCVOLCALIB_B200_H
#define LOCVOLCALIB_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define LVC_API __attribute__((visibility("default")))
#else
#define LVC_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Error codes of the generated API. */
#define FUTHARK_SUCCESS 0
#define FUTHARK_PROGRAM_ERROR 2
#define FUTHARK_OUT_OF_MEMORY 3

/* ---------------- Part 1: the generated-library API ---------------- */

struct futhark_context_config;
struct futhark_context;
struct futhark_f32_1d;
struct futhark_f64_1d;

/* lys/shared.c:20 */
LVC_API struct futhark_context_config *futhark_context_config_new(void);
/* lys/sdl/main.c:272 */
LVC_API void futhark_context_config_free(struct futhark_context_config *cfg);
/* lys/shared.c:25 -- "#N" selects CUDA device N, otherwise the first device
 * whose name contains the string. */
LVC_API void futhark_context_config_set_device(struct futhark_context_config *cfg, const char *s);
LVC_API void futhark_context_config_set_debugging(struct futhark_context_config *cfg, int flag);
LVC_API void futhark_context_config_set_profiling(struct futhark_context_config *cfg, int flag);
LVC_API void futhark_context_config_set_logging(struct futhark_context_config *cfg, int flag);
/* lys/shared.c:44 -- accepted for compatibility; the engine has no kernel
 * cache file (its kernels are compiled ahead of time for sm_100a). */
LVC_API void futhark_context_config_set_cache_file(struct futhark_context_config *cfg, const char *f);

/* Tuning parameters by name, as the generated API of a Futhark program
 * exposes them (futhark_context_config_set_tuning_param and the
 * futhark_get_tuning_param_* enumeration).  Returns 0, or 1 for an unknown
 * name or an out-of-range value.  Names:
 *   "lvc.streams"  streams a batch plan forks its launch classes over (1..8, default 4)
 *   "lvc.grid"     0: persistent grids, items taken in strides; 1: one CTA or
 *                  cluster per strike instance, handed out by the block
 *                  scheduler in descending order of work; 2 (default): 0 for
 *                  f64 plans, 1 for f32-state plans */
LVC_API int futhark_context_config_set_tuning_param(struct futhark_context_config *cfg,
                                                    const char *param_name, size_t new_value);
LVC_API int futhark_get_tuning_param_count(void);
LVC_API const char *futhark_get_tuning_param_name(int i);
LVC_API const char *futhark_get_tuning_param_class(int i);

/* lys/shared.c:47 -- returns NULL only on allocation failure; a context whose
 * device could not be initialised reports that from futhark_context_get_error. */
LVC_API struct futhark_context *futhark_context_new(struct futhark_context_config *cfg);
/* lys/sdl/main.c:271 */
LVC_API void futhark_context_free(struct futhark_context *ctx);
/* lys/sdl/main.c:109,134 -- waits for all work of the context. */
LVC_API int futhark_context_sync(struct futhark_context *ctx);
/* lys/shared.h:21-26 -- the last error message, malloc'd (caller frees), or
 * NULL if there was none; retrieving it clears it. */
LVC_API char *futhark_context_get_error(struct futhark_context *ctx);
/* Releases cached device memory of the context. */
LVC_API int futhark_context_clear_caches(struct futhark_context *ctx);

LVC_API struct futhark_f32_1d *futhark_new_f32_1d(struct futhark_context *ctx, const float *data,
                                          int64_t dim0);
LVC_API struct futhark_f64_1d *futhark_new_f64_1d(struct futhark_context *ctx, const double *data,
                                          int64_t dim0);
/* lys/sdl/main.c:131 */
LVC_API int futhark_free_f32_1d(struct futhark_context *ctx, struct futhark_f32_1d *arr);
LVC_API int futhark_free_f64_1d(struct futhark_context *ctx, struct futhark_f64_1d *arr);
/* lys/sdl/liblys.c:151 -- copies the array to host memory (synchronous). */
LVC_API int futhark_values_f32_1d(struct futhark_context *ctx, struct futhark_f32_1d *arr, float *data);
LVC_API int futhark_values_f64_1d(struct futhark_context *ctx, struct futhark_f64_1d *arr, double *data);
/* lys/shared.c:79 */
LVC_API const int64_t *futhark_shape_f32_1d(struct futhark_context *ctx, struct futhark_f32_1d *arr);
LVC_API const int64_t *futhark_shape_f64_1d(struct futhark_context *ctx, struct futhark_f64_1d *arr);

/*
 * The entry point `main` (finpar/LocVolCalib.fut:238-252; calling convention
 * of lys/sdl/main.c:108,124,130).  Prices of the strikes 0.001*i,
 * i < outer_loop_count.  The engine computes in f64 and rounds each price to
 * f32 once.  Errors: numX < 3, numY < 3, numT < 1, outer_loop_count < 0,
 * numX > 512, or an initGrid spot index outside [0, numX) (the cases where the
 * reference program fails an index or size check).
 */
LVC_API int futhark_entry_main(struct futhark_context *ctx, struct futhark_f32_1d **out0,
                       const int32_t outer_loop_count, const int32_t numX, const int32_t numY,
                       const int32_t numT, const float s0, const float t, const float alpha,
                       const float nu, const float beta);

/* ---------------- Part 2: engine extensions ---------------- */

/* `main` instantiated at f64 (what the generated library of an f64 build of
 * finpar/LocVolCalib.fut would export); same errors as futhark_entry_main. */
LVC_API int futhark_entry_main_f64(struct futhark_context *ctx, struct futhark_f64_1d **out0,
                           const int32_t outer_loop_count, const int32_t numX,
                           const int32_t numY, const int32_t numT, const double s0,
                           const double t, const double alpha, const double nu,
                           const double beta);

/* One calibration: the nine scalar inputs of `main`. */
struct lvc_calibration {
  int32_t outer, numX, numY, numT;
  double s0, t, alpha, nu, beta;
};

/* State precision of the rollback.  LVC_F64: every operation in f64.
 * LVC_F32_STATE: grid state and stencils in f32; the tridiagonal pivot
 * divisions and the payoff stay in f64. */
enum { LVC_F64 = 0, LVC_F32_STATE = 1 };

/* A batch plan: the device tables, work lists and captured CUDA graph for a
 * fixed list of calibrations.  Prices of calibration c are at offset
 * sum_{c' < c} outer[c'] of the price vector. */
struct lvc_plan;

LVC_API int lvc_plan_new(struct futhark_context *ctx, const struct lvc_calibration *calibs, int32_t n,
                 int32_t precision, struct lvc_plan **plan);
LVC_API int lvc_plan_free(struct futhark_context *ctx, struct lvc_plan *plan);
LVC_API int64_t lvc_plan_num_prices(const struct lvc_plan *plan);
/* Re-uploads the scalar inputs of a plan (sizes must be unchanged). */
LVC_API int lvc_plan_set_params(struct futhark_context *ctx, struct lvc_plan *plan,
                        const struct lvc_calibration *calibs, int32_t n);
/* Runs the whole batch (setup, pivot and rollback kernels, one graph launch)
 * asynchronously on the context's stream; prices stay in device memory. */
LVC_API int lvc_plan_run(struct futhark_context *ctx, struct lvc_plan *plan);
/* Synchronises and copies the prices to host memory (n = lvc_plan_num_prices). */
LVC_API int lvc_plan_copy_prices(struct futhark_context *ctx, struct lvc_plan *plan, double *prices);
/* Device address of the plan's price vector (valid until lvc_plan_free). */
LVC_API const double *lvc_plan_device_prices(const struct lvc_plan *plan);
/* Times `iters` back-to-back runs with CUDA events on the context stream;
 * writes the mean milliseconds per run. */
LVC_API int lvc_plan_time(struct futhark_context *ctx, struct lvc_plan *plan, int32_t iters,
                  double *ms_per_run);
/* Per-launch device time of the rollback kernel(s) of the last lvc_plan_time
 * (milliseconds, summed over the plan's rollback launches, mean per run). */
LVC_API double lvc_plan_rollback_ms(const struct lvc_plan *plan);
/* Number of kernel launches one lvc_plan_run performs. */
LVC_API int32_t lvc_plan_num_launches(const struct lvc_plan *plan);
/* One rollback launch class of a plan (no counterpart in the reference): the
 * kernel shape its instances share, their count and option-cell-steps, and
 * the class's device time in the last lvc_plan_time (mean per run, the
 * classes timed one after another on one stream). */
struct lvc_launch_info {
  int32_t family;     /* LVC_FAMILY_* */
  int32_t cluster;    /* CTAs per strike instance */
  int32_t threads;    /* threads per CTA */
  int32_t items;      /* strike instances */
  int64_t cell_steps; /* sum of numX * numY * (numT - 1) over the instances */
  double ms;          /* 0 before the first lvc_plan_time */
};
/* Number of rollback launch classes of a plan. */
LVC_API int32_t lvc_plan_num_classes(const struct lvc_plan *plan);
/* Class i (0 .. lvc_plan_num_classes - 1, largest work first); -1 when out of range. */
LVC_API int lvc_plan_launch_info(const struct lvc_plan *plan, int32_t i, struct lvc_launch_info *out);

/* One-shot batched call from host memory: plan, run, copy back, free. */
LVC_API int lvc_batch(struct futhark_context *ctx, const struct lvc_calibration *calibs, int32_t n,
              int32_t precision, double *prices);

/*
 * No counterpart in the reference.  `main` at f64 for callers that cannot
 * allocate device memory when they price (a serving loop that must not incur
 * the device-wide synchronisation of cudaMalloc/cudaFree, a host whose
 * allocator or memory budget already owns all of HBM).  Same inputs, checks
 * and errors as futhark_entry_main_f64, but the prices go to `prices`, a
 * device buffer of outer_loop_count doubles owned by the caller, and all
 * scratch comes from one static device array of LVC_NOALLOC_SCRATCH_BYTES
 * (64 MiB) that every device loading this library holds until exit -- the
 * array belongs to the library's device code, so loading the library's
 * kernels on a device reserves it whether or not this entry point is called
 * (the serving runtime's HBM budget does not count it); the call allocates no
 * device memory.  Calibrations whose scratch exceeds that size (the
 * calibration's pivot rows, about 8 * (numX + 2) * round4(numY) * (numT - 1)
 * bytes for the paired kernel, plus its tables, about 64 * numY * (numT - 1)
 * bytes; lvc_entry_main_f64_noalloc_bytes gives the exact figure; all three
 * reference datasets fit) or whose grid does not fit on chip are rejected
 * with an error.
 * The first call on each device looks up the array's device address
 * (cudaGetSymbolAddress); make that first call before any stream capture.
 * Runs on the context's stream and returns after the prices are written.
 * Every call uses the same array, so calls that overlap on the GPU (other
 * contexts or threads using this entry point at the same time) race.
 */
#define LVC_NOALLOC_SCRATCH_BYTES (64u << 20)
LVC_API int lvc_entry_main_f64_noalloc(struct futhark_context *ctx, double *prices,
                                       const int32_t outer_loop_count, const int32_t numX,
                                       const int32_t numY, const int32_t numT, const double s0,
                                       const double t, const double alpha, const double nu,
                                       const double beta);
/* No counterpart in the reference.  The scratch bytes lvc_entry_main_f64_noalloc
 * needs for a calibration of these sizes under the context's current shape
 * for the grid class (the figure it compares with LVC_NOALLOC_SCRATCH_BYTES);
 * -1 for invalid sizes or a grid that does not fit on chip.  Allocates
 * nothing. */
LVC_API int64_t lvc_entry_main_f64_noalloc_bytes(struct futhark_context *ctx, const int32_t outer_loop_count,
                                                 const int32_t numX, const int32_t numY, const int32_t numT);

/*
 * Serving runtime: continuous batching of calibration requests.  A
 * scheduler thread admits queued requests as batches -- shortest first by
 * option-cell-steps, a request queued over 50 ms first of all, no request
 * of more than 4x the work of the batch's first -- while a stream is free,
 * the in-flight request cap is not reached and the batch's tables and
 * pivots fit in what is left of the HBM budget (reserved once at creation).
 * Batches run concurrently on their own streams with one CTA (or cluster)
 * per strike instance, so SMs pass to waiting instances of any in-flight
 * batch as running ones finish; half the streams have the device's greatest
 * priority and take the batches of up to about a millisecond of GPU work.
 * Latency is measured from submit to the completion of the request's batch.
 */
struct lvc_server;
struct lvc_server_config {
  int32_t precision;              /* LVC_F64 or LVC_F32_STATE */
  int32_t max_inflight_requests;  /* 0: 256 */
  int32_t max_batch_requests;     /* 0: 64 */
  int32_t num_streams;            /* 0: 8 */
  int64_t hbm_budget_bytes;       /* 0: 8 GiB */
};
struct lvc_server_stats {
  int64_t submitted, completed, failed, options, batches, hbm_reserved_bytes;
  double p50_ms, p99_ms, mean_ms, max_ms, throughput_options_per_s, span_s;
};
LVC_API int lvc_server_new(struct futhark_context *ctx, const struct lvc_server_config *cfg,
                           struct lvc_server **server);
/* Thread-safe; invalid calibrations are rejected here with the entry
 * points' errors. */
LVC_API int lvc_server_submit(struct lvc_server *server, const struct lvc_calibration *calib,
                              uint64_t *ticket);
LVC_API int lvc_server_poll(struct lvc_server *server, uint64_t ticket, int32_t *done);
/* Blocks until the request is done (timeout_s <= 0: no limit), copies its
 * `outer` prices and releases the ticket. */
LVC_API int lvc_server_wait(struct lvc_server *server, uint64_t ticket, double *prices,
                            double timeout_s);
LVC_API int lvc_server_stats(struct lvc_server *server, struct lvc_server_stats *stats);
LVC_API int lvc_server_reset_stats(struct lvc_server *server);
/* Finishes the queued and running requests, then releases everything. */
LVC_API int lvc_server_free(struct lvc_server *server);

/* Peak probes of the context's device: FP64 FMA throughput (TFLOP/s, 2 flops
 * per FMA, every SM busy) and shared-memory load bandwidth (GB/s summed over
 * SMs), each the best of three timed microbenchmark launches.  These are the
 * two ceilings of the rollback kernel. */
LVC_API int lvc_probe_peaks(struct futhark_context *ctx, double *fp64_tflops, double *smem_gbs);

/* The cudaStream_t the context launches on (as void*). */
LVC_API void *lvc_context_stream(struct futhark_context *ctx);

/* The same tuning parameters on a live context; plans created afterwards use
 * them.  0, or FUTHARK_PROGRAM_ERROR for an unknown name or value. */
LVC_API int lvc_context_set_tuning_param(struct futhark_context *ctx, const char *param_name,
                                         size_t new_value);

/* Shape autotuner.  A grid class (numX, numY, precision) can run under
 * several shapes: kernel family x cluster size, which fix the CTA's threads,
 * rows and shared memory.  The context keeps a table of chosen shapes that
 * every plan, entry point, no-alloc call and server built from it uses;
 * classes not in the table take the built-in choice. */
#define LVC_FAMILY_CHUNK 0     /* chunked lines, any numX <= 512; grid on chip or in HBM */
#define LVC_FAMILY_LINE 1      /* one lane per grid line, any sizes with numX <= 256 */
#define LVC_FAMILY_LINE_FULL 2 /* line family on full 32 x 32 tiles (numX, rows per CTA multiples of 32) */
#define LVC_FAMILY_LINE_PAIR 3 /* full tiles walked two columns at a time (numX % 64 == 0) */
#define LVC_FAMILY_LINE_PAIR1 4 /* the same with one unit per warp: twice the warps (numX % 32 == 0) */

struct lvc_shape {
  int32_t family;       /* LVC_FAMILY_* */
  int32_t cluster;      /* CTAs per strike instance (a thread-block cluster when > 1) */
  int32_t threads;      /* threads per CTA */
  int32_t rows_per_cta; /* numY rows each CTA holds */
  int32_t smem_bytes;   /* dynamic shared memory per CTA */
  int32_t hbm_state;    /* 1: the grid lives in HBM scratch (chunk family only) */
};

struct lvc_tuning_entry {
  int32_t numX, numY, precision;
  int32_t tuned;              /* 1: chosen by lvc_autotune or set by lvc_tuning_set */
  struct lvc_shape shape;
  double us_per_step_default; /* autotune probe time of the built-in shape (0: not measured) */
  double us_per_step_best;    /* autotune probe time of the chosen shape (0: not measured) */
};

/* Every shape that can run the grid class on this device; *count receives
 * the number (entries beyond `max` are not written). */
LVC_API int lvc_shape_candidates(struct futhark_context *ctx, int32_t numX, int32_t numY,
                                 int32_t precision, struct lvc_shape *out, int32_t max,
                                 int32_t *count);
/* Pins a shape (matched on family, cluster and hbm_state) for a grid class;
 * NULL returns the class to the built-in choice. */
LVC_API int lvc_tuning_set(struct futhark_context *ctx, int32_t numX, int32_t numY,
                           int32_t precision, const struct lvc_shape *shape);
/* The shape calibration `calib` of a plan runs under (FUTHARK_PROGRAM_ERROR
 * for an index out of range). */
LVC_API int lvc_plan_shape(const struct lvc_plan *plan, int32_t calib, struct lvc_shape *out);
/* The shape the class runs under now (tuned or built-in). */
LVC_API int lvc_tuning_get(struct futhark_context *ctx, int32_t numX, int32_t numY,
                           int32_t precision, struct lvc_tuning_entry *out);
/* Entries of the table (up to `max` written); returns how many there are. */
LVC_API int32_t lvc_tuning_entries(struct futhark_context *ctx, struct lvc_tuning_entry *out,
                                   int32_t max);
/* For every grid class of the calibrations: times each candidate shape's
 * rollback on the class's own instance count (capped at 16384) for
 * probe_steps time steps (<= 0: 8), and keeps the fastest.  Synchronous. */
LVC_API int lvc_autotune(struct futhark_context *ctx, const struct lvc_calibration *calibs,
                         int32_t n, int32_t precision, int32_t probe_steps);
/* Plan-level autotuner: runs the workload's whole plan, with its time lines
 * capped at max_steps (<= 0: 32), under lvc.grid 0/1 x lvc.streams 2/4, and
 * keeps the fastest as the context's tuning parameters (reported through the
 * optional pointers, with the capped plan's time in ms).  Then, for every
 * grid class of the workload whose table shape is not the built-in one, it
 * times the plan with that class back on the built-in shape and keeps
 * whichever plan was faster.  Synchronous. */
LVC_API int lvc_autotune_plan(struct futhark_context *ctx, const struct lvc_calibration *calibs,
                              int32_t n, int32_t precision, int32_t max_steps, int32_t *grid,
                              int32_t *streams, double *ms);
/* The tuning parameters and the table as a tuning file of name=value lines:
 *   lvc.streams=4
 *   lvc.shape.f64.256x256=line_pair,8      (family: line_pair|line_pair1|line_full|line|chunk|chunk_hbm, cluster) */
LVC_API int lvc_tuning_save(struct futhark_context *ctx, const char *path);
LVC_API int lvc_tuning_load(struct futhark_context *ctx, const char *path);

#ifdef __cplusplus
}
#endif

#endif /* LOCVOLCALIB_B200_H */
