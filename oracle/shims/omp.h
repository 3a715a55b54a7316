/* ORACLE shim: libpshtlight/c_utils.c includes <omp.h> only for the thread
   count helper (c_utils.c:93); the oracle uses the generator single-threaded
   and this image's gcc has no libgomp spec, so the call is answered here. */
#ifndef ORACLE_OMP_SHIM_H
#define ORACLE_OMP_SHIM_H
static inline int omp_get_max_threads(void) { return 1; }
static inline int omp_get_thread_num(void) { return 0; }
static inline int omp_get_num_threads(void) { return 1; }
#endif
