// Ring kernels: HEALPix ring assembly + real FFTs (alm2map) and their adjoint
// (map2alm).
//
// Synthesis, per ring pair r (rings mid-r and mid+r share theta up to a sign
// of cos) and map (src/wavemoth.c:1083-1191):
//   t_m = (q_even(m, r) +- q_odd(m, r)) e^{i m phi0}
//   W[j] = sum_{m = j mod n} t_m + sum_{m > 0, m = -j mod n} conj(t_m),  j <= n/2
//   ring = unnormalised c2r_n(W)  (imaginary parts of W[0], W[n/2] ignored)
// The aliasing sum for every output bin is evaluated in increasing m, the
// order in which the reference accumulates it.
//
// The c2r of even length n = 2N runs as one complex inverse FFT of length N:
//   Z[k] = (W[k] + conj W[N-k]) + i w^k (W[k] - conj W[N-k]),  w = e^{2 pi i / n}
//   ring[2s] = Re z[s], ring[2s+1] = Im z[s],  z = IDFT_N(Z)
// and the analysis r2c uses the mirror identity.  The length-N transform is
// a mixed-radix Stockham autosort FFT in shared memory (radix 4, 2, 3, 5, 7
// butterflies in registers; any other prime factor p through a length-p DFT
// per output from the table of roots).  All twiddles come from one table of
// n-th roots of unity computed with sincospi on exact rationals.
//
// One CTA per (map, ring pair), maps fastest in the grid so that the CTAs that
// share the 32-byte sectors of q (16 bytes per map) and of the interleaved
// (npix, nmaps) map run at the same time; ring lengths are 4, 8, ..., 4 nside.
#include <cuda_runtime.h>
#include <stdint.h>

#include "plan.h"
#include "kernels.h"

namespace wm {

namespace {

constexpr int kRingThreads = 256;

struct cplx {
  double x, y;
};

__device__ __forceinline__ cplx cadd(cplx a, cplx b) { return {a.x + b.x, a.y + b.y}; }
__device__ __forceinline__ cplx csub(cplx a, cplx b) { return {a.x - b.x, a.y - b.y}; }
__device__ __forceinline__ cplx cmul(cplx a, cplx b) {
  return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
__device__ __forceinline__ cplx cconj(cplx a) { return {a.x, -a.y}; }
__device__ __forceinline__ cplx cscale(cplx a, double s) { return {a.x * s, a.y * s}; }
__device__ __forceinline__ cplx mul_i(cplx a) { return {-a.y, a.x}; }

// e^{2 pi i e / n} from the half table roots[u] = e^{2 pi i u / n}, u < n/2
__device__ __forceinline__ cplx root(const cplx *roots, int n, long long e) {
  long long u = e % n;
  if (u < 0) u += n;
  const int N = n >> 1;
  if (u < N) return roots[u];
  cplx r = roots[u - N];
  return {-r.x, -r.y};
}

__device__ __forceinline__ int pick_radix(int rem) {
  if (rem % 4 == 0) return 4;
  if (rem % 2 == 0) return 2;
  if (rem % 3 == 0) return 3;
  if (rem % 5 == 0) return 5;
  if (rem % 7 == 0) return 7;
  int p = 11;
  while (rem % p) p += 2;
  return p;
}

// Block-wide complex FFT of length N (unnormalised), sign +1: inverse
// (e^{+2 pi i jk/N}), -1: forward.  a holds the input; b is scratch of N
// entries.  Returns the buffer holding the result.  n = 2N is the length of
// the root table's circle.
__device__ cplx *block_fft(cplx *a, cplx *b, const cplx *roots, int N, int sign) {
  const int n = 2 * N;
  int rem = N, Ns = 1;
  cplx *in = a, *out = b;
  while (rem > 1) {
    const int R = pick_radix(rem);
    const int NR = N / R;
    const int tw = n / (Ns * R);
    const int rot = n / R;  // exponent unit of the radix-R DFT
    if (R <= 7) {
      for (int j = threadIdx.x; j < NR; j += blockDim.x) {
        const int k = j % Ns;
        cplx v[7];
        for (int r = 0; r < R; ++r) {
          cplx x = in[j + r * NR];
          v[r] = r ? cmul(x, root(roots, n, (long long)sign * r * k * tw)) : x;
        }
        cplx V[7];
        if (R == 2) {
          V[0] = cadd(v[0], v[1]);
          V[1] = csub(v[0], v[1]);
        } else if (R == 4) {
          cplx s02 = cadd(v[0], v[2]), d02 = csub(v[0], v[2]);
          cplx s13 = cadd(v[1], v[3]), d13 = csub(v[1], v[3]);
          cplx id = mul_i(d13);
          if (sign < 0) id = {-id.x, -id.y};
          V[0] = cadd(s02, s13);
          V[2] = csub(s02, s13);
          V[1] = cadd(d02, id);
          V[3] = csub(d02, id);
        } else if (R == 3) {
          const double c = -0.5, s = 0.86602540378443864676 * sign;
          cplx s12 = cadd(v[1], v[2]), d12 = csub(v[1], v[2]);
          cplx base = {v[0].x + c * s12.x, v[0].y + c * s12.y};
          cplx rot90 = {-s * d12.y, s * d12.x};
          V[0] = cadd(v[0], s12);
          V[1] = cadd(base, rot90);
          V[2] = csub(base, rot90);
        } else {
          for (int u = 0; u < R; ++u) {
            cplx acc = v[0];
            for (int t = 1; t < R; ++t)
              acc = cadd(acc, cmul(v[t], root(roots, n, (long long)sign * ((t * u) % R) * rot)));
            V[u] = acc;
          }
        }
        const int idxD = (j / Ns) * Ns * R + k;
        for (int r = 0; r < R; ++r) out[idxD + r * Ns] = V[r];
      }
    } else {
      // generic prime radix: twiddle in place, then one output per thread
      for (int e = threadIdx.x; e < N; e += blockDim.x) {
        const int j = e % NR, r = e / NR, k = j % Ns;
        if (r) in[e] = cmul(in[e], root(roots, n, (long long)sign * r * k * tw));
      }
      __syncthreads();
      for (int e = threadIdx.x; e < N; e += blockDim.x) {
        const int j = e % NR, u = e / NR, k = j % Ns;
        cplx acc = {0.0, 0.0};
        for (int t = 0; t < R; ++t)
          acc = cadd(acc, cmul(in[j + t * NR], root(roots, n, (long long)sign * ((t * u) % R) * rot)));
        out[(j / Ns) * Ns * R + k + u * Ns] = acc;
      }
    }
    __syncthreads();
    cplx *tmp = in;
    in = out;
    out = tmp;
    Ns *= R;
    rem /= R;
  }
  return in;
}

__device__ __forceinline__ cplx phase(int m, const DevRing &R, int enabled) {
  if (!enabled || R.phi_num == 0) return {1.0, 0.0};
  const long long den2 = 2LL * R.phi_den;
  const long long num = ((long long)m * R.phi_num) % den2;
  double s, c;
  sincospi((double)num / (double)R.phi_den, &s, &c);
  return {c, s};
}

__device__ void build_roots(cplx *roots, int n) {
  const int N = n / 2;
  for (int u = threadIdx.x; u < N; u += blockDim.x) {
    double s, c;
    sincospi((double)(2 * u) / (double)n, &s, &c);
    roots[u] = {c, s};
  }
}

__global__ void __launch_bounds__(kRingThreads) k_ring_synthesis(RingParams p) {
  extern __shared__ double smem_d[];
  cplx *sm = reinterpret_cast<cplx *>(smem_d);
  const int kmap = blockIdx.x, r = blockIdx.y;
  const DevRing R = p.rings[r];
  const int n = R.n, N = n / 2;
  cplx *bufA = sm;
  cplx *bufB = sm + (N + 1);
  cplx *roots = bufB + (N + 1);
  build_roots(roots, n);
  const int64_t qstride_m = 2LL * p.ni * p.nvecs;       // q[(2m + odd) * ni * nvecs]
  const int64_t qoff = (int64_t)r * p.nvecs + 2 * kmap;
  const int64_t half = (int64_t)p.ni * p.nvecs;
  __syncthreads();
  for (int side = 0; side < 2; ++side) {
    if (side == 1 && r == 0) break;  // the equator is written once
    const double sgn = side ? -1.0 : 1.0;
    for (int j = threadIdx.x; j <= N; j += blockDim.x) {
      cplx acc = {0.0, 0.0};
      for (int base = 0;; base += n) {
        const int m1 = base + j;
        if (m1 > p.mmax) break;
        {
          const double *qe = p.q + m1 * qstride_m + qoff;
          const double *qo = qe + half;
          cplx t = {qe[0] + sgn * qo[0], qe[1] + sgn * qo[1]};
          acc = cadd(acc, cmul(t, phase(m1, R, p.phase_shifts)));
        }
        const int m2 = base + n - j;
        if (m2 <= p.mmax) {
          const double *qe = p.q + m2 * qstride_m + qoff;
          const double *qo = qe + half;
          cplx t = {qe[0] + sgn * qo[0], qe[1] + sgn * qo[1]};
          acc = cadd(acc, cconj(cmul(t, phase(m2, R, p.phase_shifts))));
        }
      }
      bufA[j] = acc;
    }
    __syncthreads();
    for (int k = threadIdx.x; k < N; k += blockDim.x) {
      cplx Wk = bufA[k], Wc = cconj(bufA[N - k]);
      if (k == 0) {
        Wk.y = 0.0;
        Wc.y = 0.0;
      }
      cplx s = cadd(Wk, Wc), d = csub(Wk, Wc);
      bufB[k] = cadd(s, mul_i(cmul(root(roots, n, k), d)));
    }
    __syncthreads();
    cplx *res = block_fft(bufB, bufA, roots, N, +1);
    const int64_t off = side ? R.off_south : R.off_north;
    for (int s = threadIdx.x; s < N; s += blockDim.x) {
      cplx z = res[s];
      p.map[(off + 2 * s) * p.nmaps + kmap] = z.x;
      p.map[(off + 2 * s + 1) * p.nmaps + kmap] = z.y;
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kRingThreads) k_ring_analysis(RingParams p) {
  extern __shared__ double smem_d[];
  cplx *sm = reinterpret_cast<cplx *>(smem_d);
  const int kmap = blockIdx.x, r = blockIdx.y;
  const DevRing R = p.rings[r];
  const int n = R.n, N = n / 2;
  cplx *bufA = sm;
  cplx *bufB = sm + (N + 1);
  cplx *roots = bufB + (N + 1);
  build_roots(roots, n);
  const int64_t qstride_m = 2LL * p.ni * p.nvecs;
  const int64_t qoff = (int64_t)r * p.nvecs + 2 * kmap;
  const int64_t half = (int64_t)p.ni * p.nvecs;
  __syncthreads();
  for (int side = 0; side < 2; ++side) {
    if (side == 1 && r == 0) break;
    const int64_t off = side ? R.off_south : R.off_north;
    for (int s = threadIdx.x; s < N; s += blockDim.x)
      bufA[s] = {p.map_in[(off + 2 * s) * p.nmaps + kmap], p.map_in[(off + 2 * s + 1) * p.nmaps + kmap]};
    __syncthreads();
    cplx *Z = block_fft(bufA, bufB, roots, N, -1);
    cplx *F = (Z == bufA) ? bufB : bufA;
    for (int k = threadIdx.x; k <= N; k += blockDim.x) {
      cplx Zk = Z[k % N], Zc = cconj(Z[(N - k) % N]);
      cplx E = cscale(cadd(Zk, Zc), 0.5);
      cplx D = csub(Zk, Zc);
      cplx O = {0.5 * D.y, -0.5 * D.x};  // D / (2i)
      F[k] = cadd(E, cmul(cconj(root(roots, n, k)), O));
    }
    __syncthreads();
    for (int m = threadIdx.x; m <= p.mmax; m += blockDim.x) {
      const int jm = m % n;
      cplx g = jm <= N ? F[jm] : cconj(F[n - jm]);
      g = cscale(cmul(g, cconj(phase(m, R, p.phase_shifts))), p.scale);
      double *qe = p.q_out + m * qstride_m + qoff;
      double *qo = qe + half;
      if (side == 0) {
        qe[0] = g.x; qe[1] = g.y;
        qo[0] = g.x; qo[1] = g.y;
      } else {
        qe[0] += g.x; qe[1] += g.y;
        qo[0] -= g.x; qo[1] -= g.y;
      }
    }
    __syncthreads();
  }
}

}  // namespace

size_t ring_smem_bytes(int nside) {
  const size_t N = 2 * (size_t)nside;
  return (3 * N + 2) * sizeof(double) * 2;
}

cudaError_t launch_ring_synthesis(const RingParams &prm, cudaStream_t st) {
  const size_t smem = ring_smem_bytes(prm.nside);
  cudaError_t e = cudaFuncSetAttribute(k_ring_synthesis, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return e;
  dim3 grid(prm.nmaps, prm.ni);
  k_ring_synthesis<<<grid, kRingThreads, smem, st>>>(prm);
  return cudaGetLastError();
}

cudaError_t launch_ring_analysis(const RingParams &prm, cudaStream_t st) {
  const size_t smem = ring_smem_bytes(prm.nside);
  cudaError_t e = cudaFuncSetAttribute(k_ring_analysis, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return e;
  dim3 grid(prm.nmaps, prm.ni);
  k_ring_analysis<<<grid, kRingThreads, smem, st>>>(prm);
  return cudaGetLastError();
}

}  // namespace wm
