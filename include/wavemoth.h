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

#ifdef __cplusplus
}
#endif

#endif
