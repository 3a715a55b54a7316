// Strided copies of the uneven-batch graphs: the maps of several requests
// gathered into the interleaved buffers of one coalesced transform, and its
// results scattered back (batch.cpp).
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "kernels.h"

namespace wm {
namespace {

// rows x width doubles: dst[r dpitch + c] = src[r spitch + c]
__global__ void k_strided_copy(double *__restrict__ dst, int64_t dpitch, const double *__restrict__ src,
                               int64_t spitch, int64_t width, int64_t rows) {
  const int64_t n = rows * width;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = e / width, c = e - r * width;
    dst[r * dpitch + c] = src[r * spitch + c];
  }
}

}  // namespace

cudaError_t launch_strided_copy(double *dst, int64_t dpitch, const double *src, int64_t spitch, int64_t width,
                                int64_t rows, cudaStream_t st) {
  const int64_t n = rows * width;
  if (n <= 0) return cudaSuccess;
  k_strided_copy<<<(unsigned)std::min<int64_t>((n + 255) / 256, 16384), 256, 0, st>>>(dst, dpitch, src, spitch,
                                                                                        width, rows);
  return cudaGetLastError();
}

}  // namespace wm
