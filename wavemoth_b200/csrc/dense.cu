// Device FP64 Legendre seeds of the dense-recurrence (no-butterfly) plans.
//
// A dense plan holds, for every (m, parity) and ring, the three-term
// recurrence over the whole column from the first row whose value is not
// negligible: P at that row and the next (or the few values of a column
// with at most four rows left), as the reference's GPU resource format does
// (wavemoth/cuda/sht.py:20-35 get_edge, :98-148).  The values come from the
// step-1 ylmgen recurrence in l with its 2^90 rescaling
// (libpshtlight/ylmgen_c.c:643-732, restated in legendre.cuh), run here on
// the device, one thread per (m, ring):
//   k_dense_scan  finds the first l with |lambda_lm| > eps; the first row of
//                 parity p is the first k with l = m + p + 2k >= that l;
//   k_dense_fill  walks the recurrence again up to the rows the plan stores
//                 and writes them into the plan's FP64 arena.
#include <cuda_runtime.h>
#include <stdint.h>

#include "kernels.h"
#include "legendre.cuh"
#include "plan.h"

namespace wm {
namespace {

__device__ __forceinline__ int32_t parity_nk(int lmax, int m, int p) {
  return lmax - m - p >= 0 ? (lmax - m - p) / 2 + 1 : 0;
}

__global__ void k_dense_scan(int lmax, const double *__restrict__ thetas, int ni, double eps,
                             int32_t *__restrict__ kstart) {
  const int m = blockIdx.x;
  for (int r = threadIdx.x; r < ni; r += blockDim.x) {
    const int first = legendre_walk(m, thetas[r], lmax, eps, [](int, double) { return false; });
    for (int p = 0; p < 2; ++p) {
      const int32_t nk = parity_nk(lmax, m, p);
      int32_t ks = nk;
      if (first <= lmax) {
        const int d = first - m - p;
        ks = d <= 0 ? 0 : (d + 1) / 2;
        if (ks > nk) ks = nk;
      }
      kstart[(int64_t)(2 * m + p) * ni + r] = ks;
    }
  }
}

__global__ void k_dense_fill(int lmax, const double *__restrict__ thetas, int ni, double eps,
                             const int32_t *__restrict__ kstart, const DevDenseFill *__restrict__ fill,
                             double *__restrict__ f64) {
  const int m = blockIdx.x;
  for (int r = threadIdx.x; r < ni; r += blockDim.x) {
    DevDenseFill F[2];
    int32_t ks[2];
    int lstop = m - 1;  // last l this column needs
    for (int p = 0; p < 2; ++p) {
      const int64_t i = (int64_t)(2 * m + p) * ni + r;
      F[p] = fill[i];
      ks[p] = kstart[i];
      if (F[p].count > 0) lstop = max(lstop, m + p + 2 * (ks[p] + F[p].count - 1));
    }
    if (lstop < m) continue;
    legendre_walk(m, thetas[r], lmax, eps, [&](int l, double v) {
      const int p = (l - m) & 1, k = (l - m - p) >> 1, t = k - ks[p];
      if (t >= 0 && t < F[p].count) f64[F[p].base + (int64_t)t * F[p].stride] = v;
      return l < lstop;
    });
  }
}

}  // namespace

cudaError_t launch_dense_scan(int lmax, int mmax, const double *thetas, int ni, double eps, int32_t *kstart,
                              cudaStream_t st) {
  k_dense_scan<<<mmax + 1, 128, 0, st>>>(lmax, thetas, ni, eps, kstart);
  return cudaGetLastError();
}

cudaError_t launch_dense_fill(int lmax, int mmax, const double *thetas, int ni, double eps, const int32_t *kstart,
                              const DevDenseFill *fill, double *f64, cudaStream_t st) {
  k_dense_fill<<<mmax + 1, 128, 0, st>>>(lmax, thetas, ni, eps, kstart, fill, f64);
  return cudaGetLastError();
}

}  // namespace wm
