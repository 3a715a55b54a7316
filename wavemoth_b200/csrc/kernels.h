// Launch interfaces of the CUDA kernels (host side).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "plan.h"

namespace wm {

struct LegendreParams {
  const DevMatrix *mats;
  const DevDBlock *dblocks;
  const DevStrip *strips;
  const DevLevel *levels;
  const DevPair *pairs;
  const double *f64;
  const int32_t *i32;
  const int32_t *order;   // processing order of matrices (largest first)
  int32_t nmats;
  int32_t lmax;
  int32_t nvecs;          // 2 * nmaps real vectors
  int32_t ni;             // rings per hemisphere incl. equator (2 * nside)
  const double *alm_in;   // alm2map: (nalm, nvecs)
  double *alm_out;        // map2alm: (nalm, nvecs)
  const double *q_in;     // map2alm: q~ (q layout: row of (m, parity, ring) at
                          // (2m + parity) q_mstride + ring q_rstride doubles)
  double *q_out;          // alm2map: q
  int64_t q_mstride, q_rstride;
  double *scratch;        // gridDim.x slots of slot_stride doubles
  int64_t slot_stride;    // 2 * max_rows * nvecs
  int32_t *counter;       // work queue head (zeroed before launch)
  int32_t level0_given;   // alm2map: the root rows are already in each CTA's first buffer
                          // (the residual stage is skipped; trees of depth >= 1 only)
};

struct FastParams {
  const DevMatrix *mats;
  const DevPair *pairs;
  const double *f64;
  const int32_t *i32;
  const DevGroup *groups;
  const DevGCol *gcols;
  const DevTileA *tiles_a;
  const DevTileB *tiles_b;
  const DevRootUnit *roots;
  const double *seeds;     // read by the map2alm residual kernel
  double *seeds_out;       // written by the seed kernel (plan creation)
  int32_t ngroups;
  int64_t ngcols;
  int32_t ntiles_a, ntiles_b, nroots;
  int32_t max_root_k, max_root_n;
  int32_t lmax, nvecs, ni;
  const double *alm_in;    // alm2map input
  double *alm_out;         // map2alm output
  const double *q_in;      // map2alm input q~
  double *q;               // alm2map output q
  int64_t q_mstride, q_rstride;  // q row of (m, parity, ring): (2m + parity) q_mstride + ring q_rstride
  double *xbuf;            // depth-1 root blocks: X buffer (xrows x nvecs)
};

// which: 0 alm2map residual, 1 alm2map level, 2 map2alm level, 3 map2alm residual
cudaError_t launch_fast(int which, const FastParams &prm, int grid, cudaStream_t st);
cudaError_t launch_seeds(const FastParams &prm, cudaStream_t st);
int fast_vector_tiles(int nvecs);

// Split-precision residual path (legendre_split.cu).
struct SplitParams {
  const DevMatrix *mats;
  const double *f64;
  const DevGroup *groups;
  const DevGCol *gcols;
  const DevSplitGroup *sgroups;
  const DevSplitTileA *tiles_a;
  const DevSplitTileB *tiles_b;
  int32_t ngroups;
  int64_t ngcols;
  int32_t ntiles_a, ntiles_b;
  const double *seeds;            // recurrence seeds every kSeedRows rows (k_seeds)
  double2 *col_scale;             // per group column: (2^e, 2^-e) of P (alm2map)
  double2 *row_scale;             // per group row: (2^e, 2^-e) of P (map2alm)
  double2 *vec_scale;             // per group x kSplitN: scales of the alm / X operand
  int8_t *planes;                 // sliced alm / X operand chunks
  unsigned long long *colmax;     // plan creation: max |P| bits per column
  unsigned long long *rowmax;     // plan creation: max |P| bits per row
  int64_t nrowscale;
  int32_t lmax, nvecs, ni;
  int32_t v0;                     // first vector of this pass (kSplitN per pass)
  const double *alm_in;
  double *alm_out;
  const double *q_in;             // map2alm: q~
  double *q;                      // alm2map: q
  int64_t q_mstride, q_rstride;   // q row of (m, parity, ring): (2m + parity) q_mstride + ring q_rstride
  double *xbuf;
  int32_t *status;                // device status word (kStatus*)
  int64_t wait_limit;             // polls of a streamed-GEMM wait for another role (0: default)
  // level products of depth-1 roots
  const DevPair *pairs;
  const int32_t *i32;
  const DevRootUnit *roots;
  const DevSplitRoot *sroots;
  const DevSplitLevelTile *tiles_la, *tiles_lm;
  int32_t nroots, ntiles_la, ntiles_lm;
  int8_t *level_a;                // sliced W (A chunks)
  double2 *level_rs;              // row scales of W
};

// One launch of the streamed split GEMM: tiles whose A chunks were sliced
// once per plan (residual P or level W) and whose B planes come from the
// operand pre-pass of the call.
struct StreamLaunch {
  const DevStreamTile *tiles;
  const int32_t *rows;    // ntiles x kSplitM destination rows (-1: none)
  const int32_t *sidx;    // ntiles x kSplitM entries of `scales` (-1: none)
  const double2 *scales;  // (2^e, 2^-e) of the P column / P row / W row of each tile row
  const int8_t *a;        // A chunk pool
  int32_t ntiles;
  int32_t a_mn;           // 1: A chunks MN-major (map2alm residual), 0: K-major
};
cudaError_t launch_stream(const SplitParams &prm, const StreamLaunch &L, int grid, cudaStream_t st);
// Plan creation: residual P of every alm2map tile (SplitParams::tiles_a
// order, K-major chunks) and map2alm tile (tiles_b order, MN-major chunks)
// sliced into the A pools of the two launches.
cudaError_t launch_residual_slices(const SplitParams &prm, const StreamLaunch &a2m, const StreamLaunch &m2a,
                                   cudaStream_t st);

// which: 0 alm operand slices, 1 alm2map residual (P generated in the kernel),
//        2 X operand slices, 3 map2alm residual (P generated in the kernel),
//        4 alm2map level operand (X) slices, 6 map2alm level operand (q~) slices;
// the level GEMMs and the residual GEMMs on sliced P run as launch_stream.
cudaError_t launch_split(int which, const SplitParams &prm, int grid, cudaStream_t st);
// Zeroes vectors [v0, v0 + kSplitN) of the rows listed in `rows` (n entries,
// (buffer << kZeroBufShift) | row with buffer 0 q, 1 X buffer, 2 alm).
cudaError_t launch_zero_rows(const SplitParams &prm, const int64_t *rows, int32_t n, cudaStream_t st);
// Plan creation: P scales of both directions, and the sliced W of the levels.
cudaError_t launch_split_scales(const SplitParams &prm, cudaStream_t st);
cudaError_t launch_level_slices(const SplitParams &prm, cudaStream_t st);

// Dense-recurrence plans (dense.cu): first stored row of every (m, parity,
// ring) column, kstart[(2m + parity) ni + ring], for lambda_lm > eps; then
// the stored values written into the plan's FP64 arena.
cudaError_t launch_dense_scan(int lmax, int mmax, const double *thetas, int ni, double eps, int32_t *kstart,
                              cudaStream_t st);
cudaError_t launch_dense_fill(int lmax, int mmax, const double *thetas, int ni, double eps, const int32_t *kstart,
                              const DevDenseFill *fill, double *f64, cudaStream_t st);

int legendre_threads();
cudaError_t legendre_preload();
// Device address and size of the allocation-free entry point's static
// scratch array on the current device (noalloc.cu); 0 on success.
int noalloc_scratch(void **out, size_t *bytes, std::string &err);
cudaError_t launch_legendre(bool alm2map, const LegendreParams &prm, int grid, cudaStream_t st);

struct RingParams {
  const DevRing *rings;   // ni entries (ring pairs from the equator)
  int32_t ni;
  int32_t nside;
  int32_t mmax;
  int32_t nmaps;
  int32_t nvecs;
  const double *q;        // synthesis input: rows of nvecs doubles, (m, parity) of ring r at (r (mmax + 1) + m) 2 + parity
  const int32_t *ring_mend;  // per ring pair m limit (null: mmax + 1): synthesis sums m < ring_mend[r],
                             // analysis writes zero q~ rows from there on
  double *map;            // synthesis output (npix, nmaps)
  const double *map_in;   // analysis input (npix, nmaps)
  double *q_out;          // analysis output
  double scale;           // analysis: multiplies q~ (4 pi / npix for map2alm)
  double map_scale;       // synthesis: multiplies the map (1 for alm2map)
  const double *ring_weights;  // analysis: per ring pair, multiplies q~ (quadrature weights; null: 1)
  int32_t phase_shifts;   // 0 disables e^{i m phi0} (test hook)
  const double2 *twiddles;  // e^{2 pi i k / twlen}, k < twlen / 2
  int32_t twlen;
  const double *filters;  // Bluestein filter spectra (complex, bit-reversed)
  double *filters_out;    // written at plan creation
  const double2 *aux;     // Bluestein chirps and roots of unity per ring
  double *aux_out;        // written at plan creation
  int32_t max_bluestein_m;
  // CTA work list (one CTA per task, ordered by decreasing cost) and the
  // dynamic shared memory of every CTA
  const DevRingTask *tasks;
  int32_t ntasks;
  int32_t smem;           // bytes
  int32_t nphase_hi;      // entries of the coarse phase table (mmax / 64 + 1)
  // per ring pair, kPhaseLo + nphase_hi phase factors (fine then coarse
  // table), computed at plan creation
  const double2 *phases;
  double2 *phases_out;
};

// rows x width doubles from src (row pitch spitch) to dst (row pitch dpitch)
// (batch_copy.cu).
cudaError_t launch_strided_copy(double *dst, int64_t dpitch, const double *src, int64_t spitch, int64_t width,
                                int64_t rows, cudaStream_t st);

cudaError_t launch_ring_synthesis(const RingParams &prm, cudaStream_t st);
// y = a - b (n doubles), and y += x (n doubles): the steps of the iterative
// map2alm between the transforms
cudaError_t launch_residual(const double *a, const double *b, double *y, int64_t n, cudaStream_t st);
cudaError_t launch_accumulate(const double *x, double *y, int64_t n, cudaStream_t st);
// m-sharded plans: moves the 2 nvecs doubles of every (ring of this part,
// m) between the ring-side q (row (ring (mmax + 1) + m) 2 + parity, rings
// counted from the part's first) and the exchange buffer (row pair of m at
// tab[2m] + ring tab[2m + 1] doubles); gather 1: exchange -> ring side.
cudaError_t launch_shard_exchange(const int64_t *tab, int64_t nrings, int32_t mcount, int32_t nvecs,
                                  const double *src, double *dst, int gather, cudaStream_t st);
cudaError_t launch_ring_analysis(const RingParams &prm, cudaStream_t st);
cudaError_t launch_ring_setup(const RingParams &prm, double *twiddles, double *filters,
                              double *aux, double2 *phases, cudaStream_t st);
constexpr int32_t kRingPhaseLo = 64;  // fine phase table entries per ring
// Shared-memory bytes of a ring CTA whose transform buffer holds
// `buffer_cplx` complex values (transform length times lanes), with its
// phase tables.
int32_t ring_cta_smem(int64_t buffer_cplx, int32_t nphase_hi);
constexpr int32_t kRingBufferCplx = 8192;  // transform buffer of one CTA: 128 KB

}  // namespace wm
