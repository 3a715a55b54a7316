// ORACLE (test infrastructure only): host launcher for the reference's own
// GPU kernel all_transpose_legendre_transforms
// (wavemoth/cuda/legendre_transform.cu.in:643-679), compiled from the
// Tempita expansion of that template (oracle/Makefile, target refgpu).  The
// launch is the reference wrapper's: grid (mmax - mmin + 1, 2), block
// NTHREADS (wavemoth/cuda/legendre_transform.py:85-89).
#include <cuda_runtime.h>

#include REF_GPU_SOURCE

extern "C" int refgpu_nvecs(void) { return NVECS; }
extern "C" int refgpu_max_ni(void) { return MAX_NI; }

extern "C" int refgpu_all_transpose(unsigned lmax, unsigned mmin, unsigned mmax, unsigned ni, const void *resources,
                                    const double *q, double *a, void *stream) {
  if (ni > MAX_NI || mmax < mmin) return -1;
  all_transpose_legendre_transforms<<<dim3(mmax - mmin + 1, 2), dim3(NTHREADS), 0, (cudaStream_t)stream>>>(
      lmax, mmin, ni, (const char *)resources, q, a, 0);
  return (int)cudaGetLastError();
}
