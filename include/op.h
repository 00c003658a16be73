/* finpar OptionPricing on a B200: libop.so.
 *
 * Part 1 is the C API the Futhark compiler generates for
 * finpar/OptionPricing.fut (entry main, f32): configuration and context, the
 * array types of the entry point's parameters, and futhark_entry_main with
 * its output first, returning 0 or a FUTHARK_* error code with the message in
 * futhark_context_get_error.  A library of its own: the program's entry point
 * is named futhark_entry_main like LocVolCalib's.  Part 2 is an engine
 * extension on device pointers.
 *
 * The result is the mean payoff per model over num_mc_it Sobol paths, each
 * path computed in f32 in the reference's operation order; f32.exp and f32.log
 * are evaluated as the f32 rounding of the f64 function, and the sum over
 * paths is accumulated in f64 (in a fixed order) and rounded to f32 before the
 * division by num_mc_it.
 */
#ifndef LOCVOLCALIB_B200_OP_H
#define LOCVOLCALIB_B200_OP_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define OP_API __attribute__((visibility("default")))
#else
#define OP_API
#endif

#ifndef FUTHARK_SUCCESS
#define FUTHARK_SUCCESS 0
#define FUTHARK_PROGRAM_ERROR 2
#define FUTHARK_OUT_OF_MEMORY 3
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- part 1: generated API of finpar/OptionPricing.fut ---- */

struct futhark_context_config;
struct futhark_context;
struct futhark_f32_1d;
struct futhark_f32_2d;
struct futhark_f32_3d;
struct futhark_i32_2d;

OP_API struct futhark_context_config *futhark_context_config_new(void);
OP_API void futhark_context_config_free(struct futhark_context_config *cfg);
/* "#k" selects CUDA device k. */
OP_API void futhark_context_config_set_device(struct futhark_context_config *cfg, const char *s);
/* Accepted for compatibility with the generated API; no effect. */
OP_API void futhark_context_config_set_debugging(struct futhark_context_config *cfg, int flag);
OP_API void futhark_context_config_set_profiling(struct futhark_context_config *cfg, int flag);
OP_API void futhark_context_config_set_logging(struct futhark_context_config *cfg, int flag);

/* Always returns a context; when no usable sm_100 device exists every later
 * call fails with FUTHARK_PROGRAM_ERROR and futhark_context_get_error says why. */
OP_API struct futhark_context *futhark_context_new(struct futhark_context_config *cfg);
OP_API void futhark_context_free(struct futhark_context *ctx);
OP_API int futhark_context_sync(struct futhark_context *ctx);
/* The last error message (malloc'd, caller frees) or NULL; clears it. */
OP_API char *futhark_context_get_error(struct futhark_context *ctx);
OP_API int futhark_context_clear_caches(struct futhark_context *ctx);

/* Device arrays copied from row-major host data (NULL data: uninitialised). */
OP_API struct futhark_f32_1d *futhark_new_f32_1d(struct futhark_context *ctx, const float *data, int64_t dim0);
OP_API struct futhark_f32_2d *futhark_new_f32_2d(struct futhark_context *ctx, const float *data, int64_t dim0,
                                                 int64_t dim1);
OP_API struct futhark_f32_3d *futhark_new_f32_3d(struct futhark_context *ctx, const float *data, int64_t dim0,
                                                 int64_t dim1, int64_t dim2);
OP_API struct futhark_i32_2d *futhark_new_i32_2d(struct futhark_context *ctx, const int32_t *data, int64_t dim0,
                                                 int64_t dim1);
OP_API int futhark_free_f32_1d(struct futhark_context *ctx, struct futhark_f32_1d *arr);
OP_API int futhark_free_f32_2d(struct futhark_context *ctx, struct futhark_f32_2d *arr);
OP_API int futhark_free_f32_3d(struct futhark_context *ctx, struct futhark_f32_3d *arr);
OP_API int futhark_free_i32_2d(struct futhark_context *ctx, struct futhark_i32_2d *arr);
/* Copy to row-major host memory (synchronises the context's stream). */
OP_API int futhark_values_f32_1d(struct futhark_context *ctx, struct futhark_f32_1d *arr, float *data);
OP_API int futhark_values_f32_2d(struct futhark_context *ctx, struct futhark_f32_2d *arr, float *data);
OP_API int futhark_values_f32_3d(struct futhark_context *ctx, struct futhark_f32_3d *arr, float *data);
OP_API int futhark_values_i32_2d(struct futhark_context *ctx, struct futhark_i32_2d *arr, int32_t *data);
OP_API const int64_t *futhark_shape_f32_1d(struct futhark_context *ctx, struct futhark_f32_1d *arr);
OP_API const int64_t *futhark_shape_f32_2d(struct futhark_context *ctx, struct futhark_f32_2d *arr);
OP_API const int64_t *futhark_shape_f32_3d(struct futhark_context *ctx, struct futhark_f32_3d *arr);
OP_API const int64_t *futhark_shape_i32_2d(struct futhark_context *ctx, struct futhark_i32_2d *arr);

/* OptionPricing.fut:304-322.  Inputs in the entry point's order:
 * contract_number, num_mc_it, dir_vs [num_dates*num_und][num_bits] (i32),
 * md_cs [num_models][num_und][num_und], md_vols and md_drifts
 * [num_models][num_dates][num_und], md_sts [num_models][num_und], md_detvals
 * [num_models][1], md_discts [num_models][num_discts], bb_inds [3][num_dates]
 * (i32), bb_data [3][num_dates].  Output: [num_models] mean payoffs.
 * Contracts 1, 2 and 3 require (num_dates, num_und) = (1, 1), (5, 3) and
 * (367, 3) as the reference's size coercions do (:294-298); any other contract
 * prices to 0.  Errors: shapes that do not match, num_bits above 32,
 * bb_inds entries outside the dates, too few discount factors for the
 * contract. */
OP_API int futhark_entry_main(struct futhark_context *ctx, struct futhark_f32_1d **out0, int32_t contract_number,
                              int32_t num_mc_it, const struct futhark_i32_2d *dir_vs,
                              const struct futhark_f32_3d *md_cs, const struct futhark_f32_3d *md_vols,
                              const struct futhark_f32_3d *md_drifts, const struct futhark_f32_2d *md_sts,
                              const struct futhark_f32_2d *md_detvals, const struct futhark_f32_2d *md_discts,
                              const struct futhark_i32_2d *bb_inds, const struct futhark_f32_2d *bb_data);

/* ---- part 2: engine extension ---- */

/* The entry point's inputs as device pointers (row-major, the shapes above). */
struct op_args {
  int32_t contract_number, num_mc_it, num_bits, num_models, num_und, num_dates, num_discts;
  const int32_t *dir_vs;
  const float *md_cs, *md_vols, *md_drifts, *md_sts, *md_detvals, *md_discts;
  const int32_t *bb_inds;
  const float *bb_data;
};
/* Scratch (bytes, 256-byte aligned) op_price_f32 needs for these sizes. */
OP_API size_t op_scratch_bytes(struct futhark_context *ctx, const struct op_args *args);
/* Prices into out[num_models] (device), asynchronously on the context's
 * stream.  Checks shapes but not bb_inds' values (the entry point copies them
 * to the host to check them): the caller guarantees 1 <= bb_inds[0][i] <=
 * num_dates for every i, and 0 <= bb_inds[1][i] <= num_dates and
 * 1 <= bb_inds[2][i] <= num_dates for i >= 1 (the reference reads those
 * entries only). */
OP_API int op_price_f32(struct futhark_context *ctx, const struct op_args *args, float *out, void *scratch);
/* Synchronises the context's stream and reports a failed launch. */
OP_API int op_check(struct futhark_context *ctx);
/* The context's CUDA stream (a cudaStream_t). */
OP_API void *op_context_stream(struct futhark_context *ctx);
/* Order of the sum over paths (no counterpart in the reference's API; the
 * program leaves the reduce's order open, finpar/OptionPricing.fut:321).
 * OP_ORDER_F64 (the default): payoffs accumulated in f64 in a fixed tree
 * order, rounded once -- the more accurate mean.  OP_ORDER_SEQUENTIAL_F32: an
 * f32 running sum in path order, the order the reference's golden outputs
 * (the .out files of finpar/OptionPricing-data) were produced in, computed exactly; it
 * needs num_mc_it * num_models * 4 more bytes of scratch (op_scratch_bytes
 * counts them) and time for a pass over the stored payoffs.  Applies to the
 * calls that follow on this context. */
#define OP_ORDER_F64 0
#define OP_ORDER_SEQUENTIAL_F32 1
OP_API int op_context_set_reduction_order(struct futhark_context *ctx, int32_t order);

#ifdef __cplusplus
}
#endif

#endif /* LOCVOLCALIB_B200_OP_H */
