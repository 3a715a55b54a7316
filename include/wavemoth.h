/*
 * wavemoth.h -- drop-in C ABI of the Wavemoth spherical harmonic transform,
 * implemented on one NVIDIA B200 (sm_100a) by libwavemoth_b200.so.
 *
 * Every declaration below keeps the name, argument list and meaning of the
 * reference interface it replaces (src/wavemoth.h:22-46 and
 * src/wavemoth_private.h:42-142 of the reference).  Differences:
 *   - errors never abort the process: plan constructors return NULL and the
 *     reason is available from wavemoth_last_error() (include/wavemoth_b200.h);
 *     void functions record a status readable with wavemoth_plan_status();
 *   - nthreads is accepted and ignored (the work runs on the GPU);
 *   - WAVEMOTH_MEASURE / WAVEMOTH_ESTIMATE / WAVEMOTH_NO_RESOURCE_COPY are
 *     accepted and have no effect (no FFTW planning; the resource is always
 *     copied once into device memory).
 */
#ifndef WAVEMOTH_B200_WAVEMOTH_H
#define WAVEMOTH_B200_WAVEMOTH_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t bfm_index_t;                   /* src/butterfly.h.in:97 */
typedef struct _wavemoth_plan *wavemoth_plan;  /* src/wavemoth.h:18 */

#define WAVEMOTH_MMAJOR 0x0            /* src/wavemoth.h:20 */
#define WAVEMOTH_ESTIMATE 0x0          /* src/wavemoth.h:22 */
#define WAVEMOTH_MEASURE 0x1           /* src/wavemoth.h:23 */
#define WAVEMOTH_NO_RESOURCE_COPY 0x10 /* src/wavemoth.h:25 */

/* Sets the directory searched for <dir>/rev1/<Nside>.dat when a plan is
   created without a file name.  Replaces src/wavemoth.h:33 (wavemoth.c:129-135). */
void wavemoth_configure(char *resource_dir);

/* alm2map plan.  input: complex128 alm, (nalm, nmaps) C order, m-major
   (row of (l, m) = m(2 lmax - m + 3)/2 + l - m); output: float64 map
   (12 Nside^2, nmaps) C order, HEALPix RING ordering.  Both are bound at plan
   time and re-read/re-written by every wavemoth_execute.  resource_filename
   may be NULL (see wavemoth_configure).  Returns NULL on error.
   Replaces src/wavemoth.h:35-39 (wavemoth.c:383-615). */
wavemoth_plan wavemoth_plan_to_healpix(int Nside, int lmax, int mmax, int nmaps, int nthreads,
                                       double *input, double *output, int ordering,
                                       unsigned flags, char *resource_filename);

/* Replaces src/wavemoth.h:41 (wavemoth.c:837-874). */
void wavemoth_destroy_plan(wavemoth_plan plan);

/* Runs the plan's transform (blocking).  Replaces src/wavemoth.h:42
   (wavemoth.c:1271-1283). */
void wavemoth_execute(wavemoth_plan plan);

/* 2 * 2 * element_count of matrix (m, odd), the reference's flop count for
   one map.  Replaces src/wavemoth.h:44 (wavemoth.c:876-885). */
int64_t wavemoth_get_legendre_flops(wavemoth_plan plan, int m, int odd);

/* 0 and (Nside, lmax) from the file header, or -1 if the file cannot be
   opened or is shorter than its header.  Replaces src/wavemoth.h:46
   (wavemoth.c:144-155). */
int wavemoth_query_resourcefile(char *filename, int *out_Nside, int *out_lmax);

/* ---- private hooks used by the reference's tests (src/wavemoth_private.h) ---- */

/* Ring geometry; same fields as src/wavemoth_private.h:50-65. */
typedef struct {
  double *phi0s;
  bfm_index_t *ring_offsets;
  bfm_index_t nrings, mid_ring;
  bfm_index_t npix;
  int has_equator;
} wavemoth_grid_info;

/* Replaces src/wavemoth_private.h:136-137 (wavemoth.c:1199-1238). */
wavemoth_grid_info *wavemoth_create_healpix_grid_info(int Nside);
void wavemoth_free_grid_info(wavemoth_grid_info *info);

/* Phase 1 (Legendre) and phase 2 (rings + FFT) of wavemoth_execute, run
   separately on the plan's bound buffers.  Replaces
   src/wavemoth_private.h:132-134. */
void wavemoth_perform_legendre_transforms(wavemoth_plan plan);
void wavemoth_perform_backward_ffts(wavemoth_plan plan);

/* Sets every phi0 to zero (test hook).  Replaces src/wavemoth_private.h:138. */
void wavemoth_disable_phase_shifting(wavemoth_plan plan);

/* ---- kernel-level hooks (src/legendre_transform.h, src/butterfly.h.in) ----
   Host pointers throughout.  The two that compute (the Legendre transform and
   the butterfly transposed apply) run on the current CUDA device: inputs are
   copied up, one of this library's kernels runs, the output is copied back.
   Errors are reported through wavemoth_last_error() (and, for
   bfm_transpose_apply_d, its return code) instead of abort(). */

/* (alpha, beta, gamma) of the even/odd three-term recurrence for rows
   l = lmin + 2k, k = 2 .. nk-1: 3 (nk - 2) values.  Replaces
   src/legendre_transform.h:16-17 (legendre_transform.c.in:723-747). */
void wavemoth_legendre_transform_auxdata(size_t m, size_t lmin, size_t nk, double *auxdata);

/* y[i, j] = sum_{k < nk} P_k(x_i) a[2k, j] with P_0 = P[i], P_1 = Pp1[i] and
   P_k from the recurrence; a has row stride 2 nvecs (every other row is
   used), y is (nx, nvecs).  Same operations in the same order as the
   reference's scalar routine, so the same y bit for bit.  Replaces
   src/legendre_transform.h:19-26 (legendre_transform.c.in:680-716). */
void wavemoth_legendre_transform(size_t nx, size_t nl, size_t nvecs, double *a_l, double *y,
                                 double *x_squared, double *auxdata, double *P, double *Pp1);

/* The same transform with a_l in the layout of
   wavemoth_legendre_transform_pack; nvecs even; work is not used.  Replaces
   src/legendre_transform.h:28-35 (legendre_transform.c.in:640-678). */
void wavemoth_legendre_transform_sse(size_t nx, size_t nl, size_t nvecs, double *a_l, double *y,
                                     double *x_squared, double *auxdata, double *P, double *Pp1,
                                     char *work);

/* The reference's work-buffer size for the transform above (0 for
   nvecs == 2).  Replaces src/legendre_transform.h:37
   (legendre_transform.c.in:625-633). */
size_t wavemoth_legendre_transform_sse_query_work(size_t nvecs);

/* Packs rows 0, 2, 4, ... of input (row stride 2 nvecs) into the reference's
   blocked layout: rows 0-1, then chunks of 42 rows; within a chunk blocks of
   4 vectors, row after row.  Replaces src/legendre_transform.h:39-40
   (legendre_transform.c.in:330-380). */
void wavemoth_legendre_transform_pack(size_t nk, size_t nvecs, double *input, double *output);

/* Residual-block callback of the transposed apply: fill rows [start, stop)
   of buf (nvecs doubles each) from the payload.  Same type as
   src/butterfly.h.in:116-117. */
typedef void (*pull_func_t)(double *buf, size_t start, size_t stop, size_t nvecs, char *payload,
                            size_t payload_len, void *ctx);

typedef struct _bfm_plan bfm_plan;

/* Header fields of a serialized butterfly matrix; same fields as
   src/butterfly.h.in:152-155. */
typedef struct {
  size_t nrows, ncols, k_max, nblocks_max, element_count;
  size_t first_level_size, heap_size, heap_first_index;
} bfm_matrix_data_info;

/* Plan of the transposed apply (sizes only; the semaphores of the
   reference's NUMA scheduling are not used and may be NULL).  Replaces
   src/butterfly.h.in:141-143 and :144. */
bfm_plan *bfm_create_plan(size_t k_max, size_t nblocks_max, size_t nvecs, void *mem_semaphore,
                          void *cpu_semaphore);
void bfm_destroy_plan(bfm_plan *plan);

/* target (ncols, nvecs) = A^T x for the serialized butterfly matrix A at
   matrix_data (16-byte aligned), the residual blocks supplied by pull_func
   in the reference's order; 0 on success.  Replaces src/butterfly.h.in:146-151
   (butterfly.c.in:375-432). */
int bfm_transpose_apply_d(bfm_plan *plan, char *matrix_data, pull_func_t pull_func, double *target,
                          size_t target_len, void *caller_ctx);

/* Reads the 40-byte matrix header; returns the pointer just after it.
   Replaces src/butterfly.h.in:157 (butterfly.c.in:434-445). */
char *bfm_query_matrix_data(char *head, bfm_matrix_data_info *info);

/* Copies (or adds, should_add) the consecutive rows of source to the rows of
   target1 (mask entries 0 .. len1-1) and target2 (the next len2 entries)
   whose mask entry equals group; returns the mask after the last entry read.
   Replaces src/butterfly.h.in:178-184 (butterfly.c.in:57-139). */
const char *bfm_scatter(const char *mask, double *target1, double *target2, const double *source,
                        size_t len1, size_t len2, size_t nvecs, int group, int should_add);

#ifdef __cplusplus
}
#endif

#endif
