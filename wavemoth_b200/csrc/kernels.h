// Launch interfaces of the CUDA kernels (host side).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

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
  const double *q_in;     // map2alm: (2(mmax+1), ni, nvecs)
  double *q_out;          // alm2map
  double *scratch;        // gridDim.x slots of slot_stride doubles
  int64_t slot_stride;    // 2 * max_rows * nvecs
  int32_t *counter;       // work queue head (zeroed before launch)
};

int legendre_threads();
cudaError_t launch_legendre(bool alm2map, const LegendreParams &prm, int grid, cudaStream_t st);

struct RingParams {
  const DevRing *rings;   // ni entries (ring pairs from the equator)
  int32_t ni;
  int32_t nside;
  int32_t mmax;
  int32_t nmaps;
  int32_t nvecs;
  const double *q;        // synthesis input (2(mmax+1), ni, nvecs)
  double *map;            // synthesis output (npix, nmaps)
  const double *map_in;   // analysis input (npix, nmaps)
  double *q_out;          // analysis output
  double scale;           // analysis: multiplies q~ (4 pi / npix for map2alm)
  int32_t phase_shifts;   // 0 disables e^{i m phi0} (test hook)
};

size_t ring_smem_bytes(int nside);
cudaError_t launch_ring_synthesis(const RingParams &prm, cudaStream_t st);
cudaError_t launch_ring_analysis(const RingParams &prm, cudaStream_t st);

}  // namespace wm
