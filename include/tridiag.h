/* Batched tridiagonal solvers on the B200 LocVolCalib engine's contexts.
 *
 * Part 1 is the C API the Futhark compiler generates for the tridiagonal test
 * program misc/ocean-sim/tridiag-test.fut (f32 via typeinst32): its 2-D f32
 * array type and its four entry points, outputs first, then inputs, returning
 * 0 or a FUTHARK_* error code with the message in futhark_context_get_error.
 * Contexts and configurations are the ones of LocVolCalib.h.  Part 2 is an
 * engine extension (device pointers, no copies).
 *
 * Forms: tridagNested / tridagNestedConst solve each row with tridagPar
 * (misc/ocean-sim/tridiag.fut:4-79, the three scans); tridagNestedSeq /
 * tridagNestedSeqConst with tridagSeq (:81-95, normalised Thomas).  The Const
 * variants require the inner dimension INNER_DIM = 115 (tridiag-test.fut:4).
 */
#ifndef LOCVOLCALIB_B200_TRIDIAG_H
#define LOCVOLCALIB_B200_TRIDIAG_H

#include "LocVolCalib.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---- part 1: generated API of misc/ocean-sim/tridiag-test.fut ---- */

struct futhark_f32_2d;

/* A [dim0][dim1] f32 array on the device, copied from row-major host data. */
LVC_API struct futhark_f32_2d *futhark_new_f32_2d(struct futhark_context *ctx, const float *data,
                                                  int64_t dim0, int64_t dim1);
LVC_API int futhark_free_f32_2d(struct futhark_context *ctx, struct futhark_f32_2d *arr);
/* Copies the array to row-major host memory (synchronises the context's stream). */
LVC_API int futhark_values_f32_2d(struct futhark_context *ctx, struct futhark_f32_2d *arr, float *data);
LVC_API const int64_t *futhark_shape_f32_2d(struct futhark_context *ctx, struct futhark_f32_2d *arr);

/* tridiag-test.fut:14-15  map4 tridagPar over the rows of [n][m] a, b, c, y */
LVC_API int futhark_entry_tridagNested(struct futhark_context *ctx, struct futhark_f32_2d **out0,
                                       const struct futhark_f32_2d *in0, const struct futhark_f32_2d *in1,
                                       const struct futhark_f32_2d *in2, const struct futhark_f32_2d *in3);
/* tridiag-test.fut:17-18  the same with m fixed to 115 */
LVC_API int futhark_entry_tridagNestedConst(struct futhark_context *ctx, struct futhark_f32_2d **out0,
                                            const struct futhark_f32_2d *in0, const struct futhark_f32_2d *in1,
                                            const struct futhark_f32_2d *in2, const struct futhark_f32_2d *in3);
/* tridiag-test.fut:20-22  map4 tridagSeq over the rows */
LVC_API int futhark_entry_tridagNestedSeq(struct futhark_context *ctx, struct futhark_f32_2d **out0,
                                          const struct futhark_f32_2d *in0, const struct futhark_f32_2d *in1,
                                          const struct futhark_f32_2d *in2, const struct futhark_f32_2d *in3);
/* tridiag-test.fut:24-26  the same with m fixed to 115 */
LVC_API int futhark_entry_tridagNestedSeqConst(struct futhark_context *ctx, struct futhark_f32_2d **out0,
                                               const struct futhark_f32_2d *in0,
                                               const struct futhark_f32_2d *in1,
                                               const struct futhark_f32_2d *in2,
                                               const struct futhark_f32_2d *in3);

/* ---- part 2: engine extension ---- */

#define LVC_TRIDAG_SEQ 0 /* tridagSeq */
#define LVC_TRIDAG_PAR 1 /* tridagPar */

/* Solves `rows` systems of size m given as row-major [rows][m] device arrays,
 * asynchronously on the context's stream (lvc_context_stream); out may not
 * alias the inputs.  Same arithmetic as the entry points.  Any alignment of
 * the arrays is accepted; with odd m <= 256, rows a multiple of 4 and the
 * four inputs on 16-byte boundaries (as every allocation is) the inputs are
 * staged by tensor copies, the fastest path. */
LVC_API int lvc_tridag_f32(struct futhark_context *ctx, int32_t form, int64_t rows, int64_t m,
                           const float *a, const float *b, const float *c, const float *y, float *out);
/* Synchronises the context's stream and reports (FUTHARK_PROGRAM_ERROR) a
 * bounded device wait that gave up since the last check, and any CUDA error
 * of the solves.  The entry points check on every call.  (The solvers
 * themselves wait on nothing but their own asynchronous copies; the flag is
 * shared with lvc_wait_selftest.) */
LVC_API int lvc_tridag_check(struct futhark_context *ctx);
/* Self-test of the bounded mbarrier wait the rollback kernels use for their
 * bulk copies and cluster exchanges (no counterpart in the reference): one
 * warp waits at most `polls` polls (1 .. 2^22) on a fresh mbarrier that
 * nothing completes (arrive == 0) or that it completes itself first
 * (arrive != 0).  A wait that runs out raises a device flag, so this returns
 * what lvc_tridag_check reports: FUTHARK_PROGRAM_ERROR ("... timed out") for
 * arrive == 0, 0 otherwise.  The context stays usable either way. */
LVC_API int lvc_wait_selftest(struct futhark_context *ctx, int32_t polls, int32_t arrive);

#ifdef __cplusplus
}
#endif

#endif /* LOCVOLCALIB_B200_TRIDIAG_H */
