/* The turbulent-kinetic-energy step of the ocean model on a B200: libtke.so.
 *
 * Part 1 is the C API the Futhark compiler generates for
 * misc/ocean-sim/tke.fut with DTYPE = f32 (typeinst32.fut): configuration and
 * context, the array types of the entry point's parameters, and
 * futhark_entry_main with its seven outputs first and twenty-five inputs
 * after, returning 0 or a FUTHARK_* error code with the message in
 * futhark_context_get_error.  The library is separate from liblvc.so
 * because both programs' entry points are named futhark_entry_main, as two
 * Futhark-compiled programs would be.  Part 2 is an engine extension: one
 * step on caller-owned device memory, without allocations.
 *
 * Arrays are row-major: [xdim][ydim][zdim] with z innermost, [xdim][ydim],
 * and [n].  The outputs are bit for bit the reference's: every operation is
 * rounded as the reference's f32 program rounds it, in its order.
 */
#ifndef LOCVOLCALIB_B200_TKE_H
#define LOCVOLCALIB_B200_TKE_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define TKE_API __attribute__((visibility("default")))
#else
#define TKE_API
#endif

#ifndef FUTHARK_SUCCESS
#define FUTHARK_SUCCESS 0
#define FUTHARK_PROGRAM_ERROR 2
#define FUTHARK_OUT_OF_MEMORY 3
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- part 1: generated API of misc/ocean-sim/tke.fut ---- */

struct futhark_context_config;
struct futhark_context;
struct futhark_f32_1d;
struct futhark_f32_2d;
struct futhark_f32_3d;
struct futhark_i32_2d;

TKE_API struct futhark_context_config *futhark_context_config_new(void);
TKE_API void futhark_context_config_free(struct futhark_context_config *cfg);
/* "#k" selects CUDA device k. */
TKE_API void futhark_context_config_set_device(struct futhark_context_config *cfg, const char *s);
/* Accepted for compatibility with the generated API; no effect. */
TKE_API void futhark_context_config_set_debugging(struct futhark_context_config *cfg, int flag);
TKE_API void futhark_context_config_set_profiling(struct futhark_context_config *cfg, int flag);
TKE_API void futhark_context_config_set_logging(struct futhark_context_config *cfg, int flag);

/* Always returns a context; when no usable sm_100 device exists every later
 * call fails with FUTHARK_PROGRAM_ERROR and futhark_context_get_error says why. */
TKE_API struct futhark_context *futhark_context_new(struct futhark_context_config *cfg);
TKE_API void futhark_context_free(struct futhark_context *ctx);
TKE_API int futhark_context_sync(struct futhark_context *ctx);
/* The last error message (malloc'd, caller frees) or NULL; clears it. */
TKE_API char *futhark_context_get_error(struct futhark_context *ctx);
TKE_API int futhark_context_clear_caches(struct futhark_context *ctx);

/* Device arrays copied from row-major host data (NULL data: uninitialised). */
TKE_API struct futhark_f32_1d *futhark_new_f32_1d(struct futhark_context *ctx, const float *data, int64_t dim0);
TKE_API struct futhark_f32_2d *futhark_new_f32_2d(struct futhark_context *ctx, const float *data, int64_t dim0,
                                                  int64_t dim1);
TKE_API struct futhark_f32_3d *futhark_new_f32_3d(struct futhark_context *ctx, const float *data, int64_t dim0,
                                                  int64_t dim1, int64_t dim2);
TKE_API struct futhark_i32_2d *futhark_new_i32_2d(struct futhark_context *ctx, const int32_t *data, int64_t dim0,
                                                  int64_t dim1);
TKE_API int futhark_free_f32_1d(struct futhark_context *ctx, struct futhark_f32_1d *arr);
TKE_API int futhark_free_f32_2d(struct futhark_context *ctx, struct futhark_f32_2d *arr);
TKE_API int futhark_free_f32_3d(struct futhark_context *ctx, struct futhark_f32_3d *arr);
TKE_API int futhark_free_i32_2d(struct futhark_context *ctx, struct futhark_i32_2d *arr);
/* Copy to row-major host memory (synchronises the context's stream). */
TKE_API int futhark_values_f32_1d(struct futhark_context *ctx, struct futhark_f32_1d *arr, float *data);
TKE_API int futhark_values_f32_2d(struct futhark_context *ctx, struct futhark_f32_2d *arr, float *data);
TKE_API int futhark_values_f32_3d(struct futhark_context *ctx, struct futhark_f32_3d *arr, float *data);
TKE_API int futhark_values_i32_2d(struct futhark_context *ctx, struct futhark_i32_2d *arr, int32_t *data);
TKE_API const int64_t *futhark_shape_f32_1d(struct futhark_context *ctx, struct futhark_f32_1d *arr);
TKE_API const int64_t *futhark_shape_f32_2d(struct futhark_context *ctx, struct futhark_f32_2d *arr);
TKE_API const int64_t *futhark_shape_f32_3d(struct futhark_context *ctx, struct futhark_f32_3d *arr);
TKE_API const int64_t *futhark_shape_i32_2d(struct futhark_context *ctx, struct futhark_i32_2d *arr);

/* tke.fut:64-348.  Outputs (tke.fut:348): tketau, tketaup1, tketaum1,
 * dtketau, dtketaup1, dtketaum1 ([xdim][ydim][zdim]) and tke_surf_corr
 * ([xdim][ydim]).  Inputs in the entry point's order: tketau, tketaup1,
 * tketaum1, dtketau, dtketaup1, dtketaum1, utau, vtau, wtau, maskU, maskV,
 * maskW ([xdim][ydim][zdim]); dxt, dxu, dyt, dyu ([xdim], [xdim], [ydim],
 * [ydim]); dzt, dzw ([zdim]); cost, cosu ([ydim]); kbot ([xdim][ydim] i32);
 * kappaM, mxl, forc ([xdim][ydim][zdim]); forc_tke_surface ([xdim][ydim]).
 * The six 3-D state inputs are consumed (unique in the reference); the
 * outputs tketau, tketaum1, dtketaup1 and dtketaum1 share their storage with
 * the corresponding inputs, as the reference returns them unchanged.  Each
 * output must be freed; freeing an input as well is allowed. */
TKE_API int futhark_entry_main(
    struct futhark_context *ctx, struct futhark_f32_3d **out0, struct futhark_f32_3d **out1,
    struct futhark_f32_3d **out2, struct futhark_f32_3d **out3, struct futhark_f32_3d **out4,
    struct futhark_f32_3d **out5, struct futhark_f32_2d **out6, struct futhark_f32_3d *tketau,
    struct futhark_f32_3d *tketaup1, struct futhark_f32_3d *tketaum1, struct futhark_f32_3d *dtketau,
    struct futhark_f32_3d *dtketaup1, struct futhark_f32_3d *dtketaum1, const struct futhark_f32_3d *utau,
    const struct futhark_f32_3d *vtau, const struct futhark_f32_3d *wtau, const struct futhark_f32_3d *maskU,
    const struct futhark_f32_3d *maskV, const struct futhark_f32_3d *maskW, const struct futhark_f32_1d *dxt,
    const struct futhark_f32_1d *dxu, const struct futhark_f32_1d *dyt, const struct futhark_f32_1d *dyu,
    const struct futhark_f32_1d *dzt, const struct futhark_f32_1d *dzw, const struct futhark_f32_1d *cost,
    const struct futhark_f32_1d *cosu, const struct futhark_i32_2d *kbot, const struct futhark_f32_3d *kappaM,
    const struct futhark_f32_3d *mxl, const struct futhark_f32_3d *forc,
    const struct futhark_f32_2d *forc_tke_surface);

/* ---- part 2: engine extension ---- */

/* One step on device memory.  Inputs as in futhark_entry_main (the four
 * pass-through state arrays are not needed); outputs tketaup1_out, dtketau_out
 * ([xdim][ydim][zdim]) and tke_surf_corr_out ([xdim][ydim]) must not alias an
 * input; scratch holds tke_scratch_bytes(xdim, ydim, zdim) bytes on a 128-byte
 * boundary.  Asynchronous on the context's stream. */
struct tke_step_args {
  int64_t xdim, ydim, zdim;
  const float *tketau, *tketaup1, *dtketau, *dtketaum1;
  const float *utau, *vtau, *wtau, *maskU, *maskV, *maskW;
  const float *dxt, *dxu, *dyt, *dyu, *dzt, *dzw, *cost, *cosu;
  const int32_t *kbot;
  const float *kappaM, *mxl, *forc, *forc_tke_surface;
  float *tketaup1_out, *dtketau_out, *tke_surf_corr_out;
  void *scratch;
};
TKE_API size_t tke_scratch_bytes(int64_t xdim, int64_t ydim, int64_t zdim);
TKE_API int tke_step_f32(struct futhark_context *ctx, const struct tke_step_args *args);
/* Synchronises the context's stream and reports a failed step. */
TKE_API int tke_check(struct futhark_context *ctx);
/* The context's CUDA stream (a cudaStream_t). */
TKE_API void *tke_context_stream(struct futhark_context *ctx);
/* Kernel launches one step makes (for launch accounting). */
TKE_API int tke_launches_per_step(void);

#ifdef __cplusplus
}
#endif

#endif /* LOCVOLCALIB_B200_TKE_H */
