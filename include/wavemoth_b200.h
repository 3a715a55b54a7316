/*
 * wavemoth_b200.h -- entry points of libwavemoth_b200.so beyond the
 * reference's wavemoth.h: analysis (map2alm), device-pointer execution on a
 * caller's CUDA stream, error reporting and test hooks.
 *
 * Conventions: functions returning int return 0 on success and a nonzero
 * WAVEMOTH_ERR_* code otherwise; the message of the most recent failure on
 * the calling thread is returned by wavemoth_last_error().  No function
 * aborts the process.
 */
#ifndef WAVEMOTH_B200_H
#define WAVEMOTH_B200_H

#include "wavemoth.h"

#ifdef __cplusplus
extern "C" {
#endif

/* additive plan flags */
#define WAVEMOTH_DEVICE_POINTERS 0x100   /* input/output given at plan time are device pointers */
#define WAVEMOTH_PRECISION_SPLIT 0x200   /* residual products of depth-0/1 matrices as sliced int8
                                            tensor-core GEMMs re-summed in FP64 (Ozaki scheme);
                                            the recurrence, seeds and scales stay FP64 */
#define WAVEMOTH_DENSE 0x800            /* no butterfly file: every (m, parity) block as one dense
                                           three-term recurrence over all rings, seeded on the device
                                           (the reference GPU kernel's scheme, wavemoth/cuda/sht.py:20-148);
                                           resource_filename is ignored, Nside must be given */
#define WAVEMOTH_SPLIT_GENERATE 0x400    /* with WAVEMOTH_PRECISION_SPLIT: generate the residual P
                                            inside the GEMM kernels at every call instead of
                                            slicing it once per plan into device memory (6 bytes
                                            per element of the residual tiles, about 20 GB at
                                            nside 1024); the plan also falls back to this when
                                            the device lacks the memory.  Same results. */

/* status codes */
#define WAVEMOTH_OK 0
#define WAVEMOTH_ERR_ARG 1         /* invalid argument or mismatched sizes */
#define WAVEMOTH_ERR_RESOURCE 2    /* resource file missing, truncated or inconsistent */
#define WAVEMOTH_ERR_CUDA 3        /* a CUDA call failed (message has the CUDA error) */
#define WAVEMOTH_ERR_DEVICE 4      /* a kernel reported an error through its status word */
#define WAVEMOTH_ERR_NOMEM 5       /* device allocation failed or exceeds the set memory cap */

/* Message of the last failure on this thread ("" if none). */
const char *wavemoth_last_error(void);

/* Status of the last call made on the plan (WAVEMOTH_OK or an error code). */
int wavemoth_plan_status(wavemoth_plan plan);

/* Waits for `stream` (NULL: the default stream) and returns the plan's
   device status word as a status code (WAVEMOTH_ERR_DEVICE if a kernel
   recorded an expired bounded wait or a bad table entry), clearing it.
   New; device-pointer executes are asynchronous and report kernel-side
   errors only through this call. */
int wavemoth_plan_device_status(wavemoth_plan plan, void *stream);

/* map2alm plan: the analysis direction, defined as (4 pi / Npix) times the
   adjoint of alm2map (a_lm = 4pi/Npix sum_p f_p lambda_lm(theta_p)
   e^{-i m phi_p}).  Same signature as wavemoth_plan_to_healpix with the roles
   of the buffers swapped: input = map (12 Nside^2, nmaps), output = alm
   (nalm, nmaps) complex128.  No counterpart in the reference, which is
   synthesis only; the analysis-direction Legendre step there is the GPU
   prototype wavemoth/cuda/legendre_transform.cu.in:643-679. */
wavemoth_plan wavemoth_plan_from_healpix(int Nside, int lmax, int mmax, int nmaps, int nthreads,
                                         double *input, double *output, int ordering,
                                         unsigned flags, char *resource_filename);

/* Device-pointer execution on `stream` (a cudaStream_t; NULL is the CUDA
   default stream, as everywhere in the CUDA API).  Asynchronous with respect
   to the host.  The plan's
   intermediate buffers are shared by all calls on one plan, so calls on one
   plan must not overlap in time (serialise them on one stream).
   alm: (nalm, nmaps) complex128 as interleaved doubles; map: (npix, nmaps). */
int wavemoth_execute_alm2map_device(wavemoth_plan plan, const double *alm, double *map,
                                    void *stream);
int wavemoth_execute_map2alm_device(wavemoth_plan plan, const double *map, double *alm,
                                    void *stream);

/* Batches of uneven transforms as one CUDA graph launch.  New; the
   reference executes one plan at a time (src/wavemoth.c:1271-1283).
   Request i runs plans[i] in directions[i] (0 alm2map, 1 map2alm) from the
   device buffer inputs[i] into outputs[i]; the plans may differ in nside,
   lmax, nmaps and precision, but no two requests may share a plan.  At
   creation waits for `stream`, captures the requests, longest first, onto
   1, 2, 4 or 8 (at most max_width; <= 0 for 8) parallel graph branches,
   times each graph on a private stream (this runs every request a few
   times) and keeps the fastest.  Requests of one direction whose plans
   share a device image (same plan file, lmax, precision and settings,
   device pointers, no ring weights) run as one transform of their summed
   map count, on a plan and interleaved buffers the batch allocates here and
   frees with it; the graph gathers their inputs and scatters the results,
   which equal those of the separate calls.  Creation must not run inside
   another stream capture. */
typedef struct _wavemoth_batch *wavemoth_batch;
wavemoth_batch wavemoth_batch_create(int nreq, const wavemoth_plan *plans, const int *directions,
                                     const double *const *inputs, double *const *outputs,
                                     int max_width, void *stream);
/* One graph launch of every request of the batch on `stream`. */
int wavemoth_batch_execute(wavemoth_batch batch, void *stream);

/* wavemoth_batch_create with an explicit schedule search: schedules[2 k] =
   parallel graph branches, schedules[2 k + 1] = SMs per request for the
   persistent Legendre kernels (0: all; applied to every request when there
   is more than one branch), k < nschedules.  Every schedule is captured and
   timed, the fastest kept (one schedule: no timing).  The chosen one is
   reported by wavemoth_batch_schedule. */
wavemoth_batch wavemoth_batch_create_scheduled(int nreq, const wavemoth_plan *plans, const int *directions,
                                               const double *const *inputs, double *const *outputs,
                                               const int *schedules, int nschedules, void *stream);
int wavemoth_batch_schedule(wavemoth_batch batch, int *width, int *sms, double *ms);
/* The branch count the creation chose and its measured time per launch. */
int wavemoth_batch_info(wavemoth_batch batch, int *width, double *ms);
/* Transforms the batch's graph runs after coalescing (<= the requests). */
int wavemoth_batch_transforms(wavemoth_batch batch);
void wavemoth_batch_destroy(wavemoth_batch batch);

/* The alm2map Legendre step of `plan` (q = A^T a for every (m, parity)),
   for callers that cannot allocate device memory when they run it (inside a
   custom allocator's callback, under a framework that owns all device
   memory, or while other latency-critical work must not see driver
   allocations).  alm: device input as for wavemoth_execute_alm2map_device;
   q: device output of 2 (mmax+1) * 2 Nside * 2 nmaps doubles in the layout
   of wavemoth_get_work.  The kernel's level buffers come from one 32 MiB
   static device array that the library holds on every GPU that loads it
   until the process exits; nothing is allocated or freed by this call.
   Problems whose per-CTA buffers (2 x largest level x 2 nmaps doubles) do
   not fit are rejected with WAVEMOTH_ERR_NOMEM; smaller ones run on as many
   CTAs as fit.  The array's device address is looked up
   (cudaGetSymbolAddress) when a plan is created on a device, which loads
   the module holding the array: the 32 MiB are taken then, together with
   the code of the kernel this call launches, so the call itself makes the
   driver allocate nothing.  The kernel is the generic FP64 butterfly kernel
   over every (m, parity) matrix, so q agrees with the plan's own path to
   rounding.  All calls share the array and its contents persist between
   calls: calls that overlap on the GPU race, so serialise them.  No
   counterpart in the reference. */
int wavemoth_legendre_alm2map_noalloc(wavemoth_plan plan, const double *alm, double *q,
                                      void *stream);

/* Copies the Legendre-phase output q (complex128, (mmax+1, 2, 2 Nside, nmaps))
   to host memory `out`; the analogue of ShtPlan.get_work
   (wavemoth/lib.pyx:158-179). */
int wavemoth_get_work(wavemoth_plan plan, double *out);

/* Plan geometry queries. */
int wavemoth_plan_nmaps(wavemoth_plan plan);
int wavemoth_plan_nside(wavemoth_plan plan);
int wavemoth_plan_lmax(wavemoth_plan plan);
/* Device bytes held by the plan (program arena + buffers). */
int64_t wavemoth_plan_device_bytes(wavemoth_plan plan);
/* Bytes of the compiled butterfly program (interpolants, recurrence data). */
int64_t wavemoth_plan_program_bytes(wavemoth_plan plan);
/* Bytes of the plan's device image: the data that does not depend on the
   number of maps (program, tensor-core and split tables, sliced P and W,
   ring tables).  Plans made from the same resource file (same path, size
   and modification time), lmax, mmax and precision flags share one image;
   it is freed with the last of them.  Included in
   wavemoth_plan_device_bytes. */
int64_t wavemoth_plan_image_bytes(wavemoth_plan plan);

/* Caps the device memory a plan may allocate (bytes; <= 0 removes the cap).
   Plans whose buffers would exceed it fail with WAVEMOTH_ERR_NOMEM.  Used to
   exercise allocation-failure handling without exhausting the GPU. */
void wavemoth_set_device_memory_cap(int64_t bytes);

/* The Legendre phase alone on device buffers, q in this library's layout
   (rows of 2 nmaps doubles, (m, parity) of ring pair r at row
   (r (mmax + 1) + m) 2 + parity): q = Lambda a for every (m, parity)
   (alm2map), a = Lambda^T q (map2alm; no 4 pi / Npix, which the ring
   analysis applies).  The device-buffer analogue of
   wavemoth_perform_legendre_transforms (src/wavemoth_private.h:132). */
int wavemoth_legendre_alm2map_device(wavemoth_plan plan, const double *alm, double *q, void *stream);
int wavemoth_legendre_map2alm_device(wavemoth_plan plan, const double *q, double *alm, void *stream);

/* ---- m-sharded transforms over several GPUs (one process per GPU) ----
   Part `part` of `nparts` (every process makes the same call with its own
   part): the Legendre step for a contiguous range of m (ranges balanced by
   the matrices' estimated work) and the ring FFTs for a contiguous range of
   ring pairs (balanced by pixels), with one all-to-all of q between them.
   Device pointers, caller streams; the exchange itself is the caller's
   (NCCL all-to-all; wavemoth_b200.shard.ShardedTransform does it with
   torch.distributed).  Buffers, with nvecs = 2 nmaps, R_k = ring pairs and
   M_k = m values of part k, this part p:
     q_send (alm2map) / q_recv (map2alm): Legendre side,
         [ring 0 .. 2 Nside)[m in M_p][parity][nvecs];
     q_recv (alm2map) / q_send (map2alm): exchange side,
         [part k][ring in R_p][m in M_k][parity][nvecs];
     q_ring: ring side scratch, [ring in R_p][m 0 .. mmax][parity][nvecs].
   alm2map: legendre (alm -> q_send), all-to-all (q_send block of part k =
   its rings, in order), rings (q_recv -> the map's pixels of R_p).
   map2alm: rings (map -> q_send, block of part k = its m), all-to-all,
   legendre (q_recv -> alm rows of M_p).  New: the reference splits m over
   threads of one host (src/wavemoth.c:496-552), not over devices. */
wavemoth_plan wavemoth_plan_shard(int Nside, int lmax, int mmax, int nmaps, unsigned flags,
                                  char *resource_filename, int nparts, int part);
/* m_bounds[k] .. m_bounds[k + 1] and ring_bounds[k] .. ring_bounds[k + 1]
   are part k's ranges (nparts + 1 entries each). */
int wavemoth_shard_layout(wavemoth_plan plan, int64_t *m_bounds, int64_t *ring_bounds);
int wavemoth_shard_alm2map_legendre(wavemoth_plan plan, const double *alm, double *q_send, void *stream);
int wavemoth_shard_alm2map_rings(wavemoth_plan plan, const double *q_recv, double *q_ring, double *map,
                                 void *stream);
int wavemoth_shard_map2alm_rings(wavemoth_plan plan, const double *map, double *q_ring, double *q_send,
                                 void *stream);
int wavemoth_shard_map2alm_legendre(wavemoth_plan plan, const double *q_recv, double *alm, void *stream);

/* Quadrature weights of the analysis direction: weights[r] (r = 0 .. 2 Nside
   - 1, ring pairs from the equator; positive) multiplies the pixels of the
   rings mid - r and mid + r in map2alm, a_lm = 4 pi / Npix sum_p w_r(p) f_p
   lambda_lm(theta_p) e^{-i m phi_p}.  NULL restores unit weights.  Host
   pointer; copied.  The alm2map direction is unchanged.  New: the reference
   has no analysis direction. */
int wavemoth_plan_set_ring_weights(wavemoth_plan plan, const double *weights);

/* map2alm refined by niter Jacobi iterations, a_{k+1} = a_k +
   map2alm(f - alm2map(a_k)), on device buffers (layouts as
   wavemoth_execute_map2alm_device) on `stream`.  The first call with
   niter > 0 allocates two plan-owned buffers (a map and an alm).  With ring
   weights set, every map2alm of the iteration is weighted.  New. */
int wavemoth_map2alm_iterative_device(wavemoth_plan plan, const double *map, double *alm, int niter,
                                      void *stream);

/* The adjoint of the plan's transform on its bound buffers: reads the
   output buffer, writes the input buffer.  alm2map plan: alm = (Npix / 4 pi)
   map2alm(map); map2alm plan: map = (4 pi / Npix) alm2map(alm) -- the
   adjoints with respect to the real inner product on maps and
   <a, b> = sum_lm c_m Re(a_lm conj b_lm), c_0 = 1, c_m = 2, on alm.  Status
   through wavemoth_plan_status.  New: the reference has no analysis
   direction (src/wavemoth.c:1271-1283 is synthesis only). */
void wavemoth_execute_adjoint(wavemoth_plan plan);

/* Caps the SMs the plan's persistent Legendre kernels (the tensor-core and
   split GEMMs, which walk the plan's (m, parity) tile list) may occupy; 0
   restores all.  Used by the batch scheduler so that concurrent requests
   share the GPU; results do not depend on it. */
int wavemoth_plan_set_grid_cap(wavemoth_plan plan, int sms);

/* Test hook: how many times a wait of the streamed split-precision GEMM
   (wavemoth_execute_*_device with WAVEMOTH_PRECISION_SPLIT) polls its
   mbarrier for another warp role before it gives up (0 restores the
   default, about a second).  A wait that gives up records a timeout in the
   plan's device status word, which wavemoth_plan_device_status reports as
   WAVEMOTH_ERR_DEVICE; the kernel then
   waits for the copies and MMAs it already issued, frees its tensor memory
   and returns, so the context stays usable.  With a tiny limit a call
   fails this way on purpose.  New; it replaces the reference's abort() on a
   failed check (src/wavemoth_error.h:1-19). */
int wavemoth_plan_set_wait_limit(wavemoth_plan plan, int64_t polls);

/* Per-kernel device timing of a plan, from CUDA events recorded on the
   launching stream.  mode 1: reset and enable, 0: reset and disable,
   2: read into out[8] = (ms Legendre alm2map, ms Legendre map2alm, ms ring
   synthesis, ms ring analysis, and the four launch counts); reading waits
   for the recorded events. */
int wavemoth_plan_timing(wavemoth_plan plan, int mode, double *out);

/* Test hook: one_side = 1 makes the ring kernels run the two hemispheres of
   every ring pair one after the other within a CTA (the layout used for
   transforms longer than 4096 points, nside 2048), 0 restores the default
   (both hemispheres at once where they fit).  Results are the same. */
int wavemoth_plan_set_hemisphere_mode(wavemoth_plan plan, int one_side);

/* Number of this library's kernels launched by the plan's executes since the
   last wavemoth_plan_timing reset (mode 0 or 1); -1 for a NULL plan. */
int64_t wavemoth_plan_kernel_launches(wavemoth_plan plan);

/* Algorithmic work of one transform direction of the plan for nmaps maps:
   out[0] Legendre flops (2 per multiply-add, 5 per recurrence step),
   out[1] compressed-matrix bytes read, out[2] alm + q bytes of one Legendre
   launch, out[3] q + map bytes of one ring launch, out[4..6] interpolation /
   recurrence / dense residual element counts, out[7] Legendre grid size,
   and for the split-precision residual products (out needs 12 entries):
   out[8] / out[9] elements of P generated by the alm2map / map2alm tiles
   per pass of 64 vectors (zero padding of the tiles included), out[10] /
   out[11] int8 tensor-core operations of one alm2map / map2alm launch
   (residual and level GEMMs). */
int wavemoth_plan_work(wavemoth_plan plan, int nmaps, double *out);

/* Parses and validates a rev1 file for (Nside, lmax) exactly as plan
   creation does, without touching the GPU.  On success returns 0 and, if
   out_stats is not NULL, fills out_stats[0..7] = (matrices, residual blocks,
   strips, levels, interpolation pairs, f64 arena bytes, i32 arena bytes,
   largest intermediate buffer rows).  No counterpart in the reference. */
int wavemoth_check_resourcefile(char *filename, int Nside, int lmax, int64_t *out_stats);

/* Host-side numerical tools of the plan-file writer (no GPU needed). */
int wm_host_legendre(int m, const double *theta, int ntheta, int lmax, double eps, double *out);
void wm_host_recurrence_coefficients(int64_t m, int64_t lmin, int64_t nk, double *aux);
void wm_host_recurrence_last_row(const double *x2, const double *P0, const double *P1, const double *aux,
                                 int64_t nx, int64_t nk, double *out);
int wm_host_interp_decomp(double *A, int m, int n, double eps, int *krank, int *perm,
                          double *proj);

#ifdef __cplusplus
}
#endif

#endif
