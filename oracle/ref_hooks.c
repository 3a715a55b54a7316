/*
 * ORACLE (test infrastructure only): glue compiled together with the
 * reference's own C sources into oracle/_ref/libwavemoth_ref.so.
 *
 *  1. FFTW3 entry points (declared in shims/fftw3.h) backed by oracle/fft.c.
 *  2. libnuma entry points (shims/numa.h).  Every usable CPU is presented as
 *     a NUMA node of its own (at most 8: src/wavemoth_private.h node_plans[8]).
 *     With two or more CPUs on one node the reference's plan creation reduces
 *     the per-node buffer sizes k_max / nblocks_max across threads with its
 *     barriers commented out (src/wavemoth.c:766-783), and the thread that
 *     first faults the resource in (icpu == 0, :690-727) resets the shared
 *     value after the others have contributed; the workers then get buffers
 *     that are too small and the reference's own assert
 *     (src/butterfly.c.in:341) aborts.  One CPU per node is the only
 *     configuration in which the unmodified reference plans reliably.
 *  3. Read-only accessors for plan internals that the reference's Cython
 *     layer reads directly: the Legendre-phase output work_q
 *     (wavemoth/lib.pyx:158-179, ShtPlan.get_work) and the phi0 table
 *     (wavemoth/lib.pyx:203-213).
 */
#define _GNU_SOURCE
#include <sched.h>
#include <stdlib.h>
#include <string.h>
#include <complex.h>
#include <semaphore.h>
#include <pthread.h>
#include "wavemoth_private.h"
#include "numa.h"

/* ---------------- FFTW3 shim ---------------- */
typedef struct or_fft_plan or_fft_plan;
or_fft_plan *or_fft_plan_create(int n);
void or_fft_plan_destroy(or_fft_plan *p);
void or_fft_c2r_many(or_fft_plan *p, int howmany, const double *in, int istride,
                     int idist, double *out, int ostride, int odist);

struct or_fftw_plan_s {
  or_fft_plan *fft;
  int n, howmany, istride, idist, ostride, odist;
};

fftw_plan fftw_plan_many_dft_c2r(int rank, const int *n, int howmany,
                                 fftw_complex *in, const int *inembed,
                                 int istride, int idist, double *out,
                                 const int *onembed, int ostride, int odist,
                                 unsigned flags) {
  (void)in; (void)inembed; (void)out; (void)onembed; (void)flags;
  if (rank != 1) return NULL;
  struct or_fftw_plan_s *p = calloc(1, sizeof(*p));
  p->fft = or_fft_plan_create(n[0]);
  p->n = n[0]; p->howmany = howmany;
  p->istride = istride; p->idist = idist; p->ostride = ostride; p->odist = odist;
  return p;
}

void fftw_execute_dft_c2r(const fftw_plan p, fftw_complex *in, double *out) {
  /* a plan keeps one scratch buffer; the reference executes each ring plan
     from a single thread, so no locking is needed */
  or_fft_c2r_many(p->fft, p->howmany, (const double *)in, p->istride, p->idist,
                  out, p->ostride, p->odist);
}

void fftw_destroy_plan(fftw_plan p) {
  if (!p) return;
  or_fft_plan_destroy(p->fft);
  free(p);
}

/* ---------------- libnuma shim ---------------- */
#define OR_MASK_BITS 1024
#define OR_CPUS_PER_NODE 1

static int or_cpus[OR_MASK_BITS];
static int or_ncpus = -1;
static int or_cpu_limit = 0;

static void or_init_cpus(void) {
  if (or_ncpus >= 0) return;
  cpu_set_t set;
  or_ncpus = 0;
  if (sched_getaffinity(0, sizeof(set), &set) == 0) {
    for (int c = 0; c < CPU_SETSIZE && c < OR_MASK_BITS; ++c)
      if (CPU_ISSET(c, &set)) {
        if (or_cpu_limit > 0 && or_ncpus >= or_cpu_limit) break;
        or_cpus[or_ncpus++] = c;
      }
  }
  if (or_ncpus == 0) { or_cpus[0] = 0; or_ncpus = 1; }
}

/* Present exactly n CPUs (the plan's nthreads) so that every presented node
   owns at least one thread: the reference hands m values round-robin to all
   presented nodes (src/wavemoth.c:496-508) and only that node's threads drain
   its queue. */
void refhook_set_ncpus(int n) { or_cpu_limit = n; or_ncpus = -1; }

static int or_nnodes(void) {
  or_init_cpus();
  int n = (or_ncpus + OR_CPUS_PER_NODE - 1) / OR_CPUS_PER_NODE;
  return n > 8 ? 8 : n;
}

static struct bitmask *or_mask_new(void) {
  struct bitmask *b = malloc(sizeof(*b));
  b->size = OR_MASK_BITS;
  b->maskp = calloc(OR_MASK_BITS / (8 * sizeof(unsigned long)), sizeof(unsigned long));
  return b;
}

struct bitmask *numa_allocate_nodemask(void) { return or_mask_new(); }
struct bitmask *numa_allocate_cpumask(void) { return or_mask_new(); }
void numa_free_nodemask(struct bitmask *b) { if (b) { free(b->maskp); free(b); } }
void numa_free_cpumask(struct bitmask *b) { numa_free_nodemask(b); }

int numa_bitmask_isbitset(const struct bitmask *b, unsigned int n) {
  if (n >= b->size) return 0;
  return (b->maskp[n / (8 * sizeof(unsigned long))] >> (n % (8 * sizeof(unsigned long)))) & 1UL;
}
struct bitmask *numa_bitmask_setbit(struct bitmask *b, unsigned int n) {
  if (n < b->size) b->maskp[n / (8 * sizeof(unsigned long))] |= 1UL << (n % (8 * sizeof(unsigned long)));
  return b;
}
struct bitmask *numa_bitmask_clearbit(struct bitmask *b, unsigned int n) {
  if (n < b->size) b->maskp[n / (8 * sizeof(unsigned long))] &= ~(1UL << (n % (8 * sizeof(unsigned long))));
  return b;
}
struct bitmask *numa_bitmask_clearall(struct bitmask *b) {
  memset(b->maskp, 0, b->size / 8);
  return b;
}
unsigned int numa_bitmask_nbytes(struct bitmask *b) { return b->size / 8; }

static struct bitmask *or_all_nodes(void) {
  struct bitmask *b = or_mask_new();
  for (int i = 0; i < or_nnodes(); ++i) numa_bitmask_setbit(b, i);
  return b;
}
struct bitmask *numa_get_run_node_mask(void) { return or_all_nodes(); }
struct bitmask *numa_get_membind(void) { return or_all_nodes(); }
void numa_set_membind(struct bitmask *b) { (void)b; }
int numa_max_node(void) { return or_nnodes() - 1; }

int numa_node_to_cpus(int node, struct bitmask *mask) {
  or_init_cpus();
  numa_bitmask_clearall(mask);
  int nn = or_nnodes();
  for (int i = 0; i < or_ncpus; ++i)
    if (i % nn == node) numa_bitmask_setbit(mask, or_cpus[i]);
  return 0;
}

void *numa_alloc_onnode(size_t size, int node) { (void)node; return calloc(1, size); }
void numa_free(void *mem, size_t size) { (void)size; free(mem); }
int numa_move_pages(int pid, unsigned long count, void **pages, const int *nodes,
                    int *status, int flags) {
  (void)pid; (void)count; (void)pages; (void)nodes; (void)status; (void)flags;
  return 0;
}

/* ---------------- plan accessors ---------------- */

/* Copy the Legendre-phase buffers into out[(m*2 + odd)*nrings_half*nvecs +
   ring*nvecs + v], the layout of ShtPlan.get_work (wavemoth/lib.pyx:158-179). */
void refhook_get_work(wavemoth_plan plan, double *out) {
  size_t nrings_half = plan->grid->mid_ring + 1;
  size_t nvecs = 2 * plan->nmaps;
  size_t stride = plan->work_q_stride;
  for (int inode = 0; inode < plan->nnodes; ++inode) {
    wavemoth_node_plan_t *np = plan->node_plans[inode];
    for (size_t im = 0; im < np->nm; ++im) {
      size_t m = np->m_resources[im].m;
      for (int odd = 0; odd < 2; ++odd) {
        memcpy(out + (m * 2 + odd) * nrings_half * nvecs,
               np->work_q + (2 * im + odd) * stride,
               sizeof(double) * nrings_half * nvecs);
      }
    }
  }
}

int refhook_ncpus_total(wavemoth_plan plan) { return plan->ncpus_total; }

int refhook_phi0s(int Nside, double *out) {
  wavemoth_grid_info *g = wavemoth_create_healpix_grid_info(Nside);
  int n = g->nrings;
  for (int i = 0; i < n; ++i) out[i] = g->phi0s[i];
  wavemoth_free_grid_info(g);
  return n;
}

/* The driver loop of compute_normalized_associated_legendre
   (wavemoth/legendre.pyx:64-98) over the reference's own generator:
   out is (ntheta, lmax - m + 1). */
#include "ylmgen_c.h"
int refhook_legendre(int m, const double *theta, int ntheta, int lmax, double epsilon,
                     double *out) {
  Ylmgen_C ctx;
  int nl = lmax - m + 1;
  if (lmax < m) return -1;
  Ylmgen_init(&ctx, lmax, lmax, 0, 0, epsilon);
  Ylmgen_set_theta(&ctx, theta, ntheta);
  for (int row = 0; row < ntheta; ++row) {
    Ylmgen_prepare(&ctx, row, m);
    Ylmgen_recalc_Ylm(&ctx);
    int firstl = ctx.firstl[0];
    for (int col = m; col < (firstl < lmax + 1 ? firstl : lmax + 1); ++col)
      out[(size_t)row * nl + col - m] = 0;
    for (int col = (m > firstl ? m : firstl); col < lmax + 1; ++col)
      out[(size_t)row * nl + col - m] = ctx.ylm[col];
  }
  Ylmgen_destroy(&ctx);
  return 0;
}

/* 1 if every Legendre worker's buffers (k_max, nblocks_max) are at least
   the largest the matrices of its NUMA node need, else 0.
   wavemoth_plan_to_healpix reduces these per node across the node's threads
   without a barrier (src/wavemoth.c:766-783, barriers commented out); callers
   recreate the plan when this returns 0 instead of letting the reference's
   assert (src/butterfly.c.in:341) abort the process. */
int refhook_worker_sizes_ok(wavemoth_plan plan) {
  for (int inode = 0; inode < plan->nnodes; ++inode) {
    wavemoth_node_plan_t *np = plan->node_plans[inode];
    size_t need_k = 0, need_b = 0;
    for (size_t im = 0; im < np->nm; ++im) {
      for (int odd = 0; odd < 2; ++odd) {
        bfm_matrix_data_info info;
        bfm_query_matrix_data(np->m_resources[im].data[odd], &info);
        if (info.k_max > need_k) need_k = info.k_max;
        if (info.nblocks_max > need_b) need_b = info.nblocks_max;
      }
    }
    for (int icpu = 0; icpu < np->ncpus; ++icpu) {
      bfm_plan *b = np->cpu_plans[icpu].legendre_workers[0].bfm;
      if (b->k_max < need_k || b->nblocks_max < need_b) return 0;
    }
  }
  return 1;
}
