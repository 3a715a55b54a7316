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
// and the analysis r2c uses the mirror identity.
//
// Length-N transforms, in place in one shared-memory buffer:
//   * N a power of two (every belt ring): radix-2 Cooley-Tukey.  The inverse
//     reads its input in bit-reversed order (Z is stored there as it is
//     formed) and writes natural order; the forward (decimation in
//     frequency) reads natural order and leaves the spectrum bit-reversed.
//   * any other N (polar rings, n = 4i): Bluestein's chirp-z identity
//     jk = (j^2 + k^2 - (k - j)^2) / 2 turns the DFT into a cyclic convolution
//     of length M = 2^p >= 2N - 1: forward decimation-in-frequency FFT of the
//     chirped input (bit-reversed spectrum), product with the chirp filter's
//     spectrum (precomputed per ring at plan creation, stored bit-reversed),
//     inverse decimation-in-time FFT back to natural order.
// Twiddles come from one table of e^{2 pi i k / TW}, TW the largest power of
// two used, computed with sincospi on exact rationals; chirps and the w^k of
// the real-input identity likewise.
//
// One CTA per (map, ring pair), maps fastest in the grid so that the CTAs that
// share the 32-byte sectors of q (16 bytes per map) and of the interleaved
// (npix, nmaps) map run at the same time.
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

__device__ __forceinline__ unsigned bitrev(unsigned k, int bits) {
  return bits ? (__brev(k) >> (32 - bits)) : 0u;
}

// e^{sign 2 pi i j / len}, j < len/2, from tw[k] = e^{2 pi i k / TW}
__device__ __forceinline__ cplx twiddle(const double2 *tw, int twlen, int len, int j, int sign) {
  const double2 t = tw[(int64_t)j * (twlen / len)];
  return {t.x, sign * t.y};
}

__device__ __forceinline__ int ilog2(int v) { return 31 - __clz(v); }

// In-place forward (sign -1) or inverse (+1) DIF: natural in, bit-reversed
// out.  Consecutive radix-2 stages (len, len/2) are fused into one pass over
// the data (radix 2^2), which leaves the output order unchanged.
__device__ void fft_dif(cplx *x, int M, const double2 *tw, int twlen, int sign) {
  int len = M;
  for (; len >= 4; len >>= 2) {
    const int q = len >> 2;
    for (int b = threadIdx.x; b < M / 4; b += blockDim.x) {
      const int j = b % q, base = (b / q) * len + j;
      const cplx a0 = x[base], a1 = x[base + q], a2 = x[base + 2 * q], a3 = x[base + 3 * q];
      const cplx w1 = twiddle(tw, twlen, len, j, sign), w1b = twiddle(tw, twlen, len, j + q, sign);
      const cplx w2 = twiddle(tw, twlen, len >> 1, j, sign);
      const cplx b0 = cadd(a0, a2), b2 = cmul(csub(a0, a2), w1);
      const cplx b1 = cadd(a1, a3), b3 = cmul(csub(a1, a3), w1b);
      x[base] = cadd(b0, b1);
      x[base + q] = cmul(csub(b0, b1), w2);
      x[base + 2 * q] = cadd(b2, b3);
      x[base + 3 * q] = cmul(csub(b2, b3), w2);
    }
    __syncthreads();
  }
  if (len == 2) {
    for (int b = threadIdx.x; b < M / 2; b += blockDim.x) {
      const cplx u = x[2 * b], v = x[2 * b + 1];
      x[2 * b] = cadd(u, v);
      x[2 * b + 1] = csub(u, v);
    }
    __syncthreads();
  }
}

// In-place DIT: bit-reversed in, natural out; stages (L, 2L) fused.
__device__ void fft_dit(cplx *x, int M, const double2 *tw, int twlen, int sign) {
  int L = 2;
  if (ilog2(M) & 1) {
    for (int b = threadIdx.x; b < M / 2; b += blockDim.x) {
      const cplx u = x[2 * b], v = x[2 * b + 1];
      x[2 * b] = cadd(u, v);
      x[2 * b + 1] = csub(u, v);
    }
    __syncthreads();
    L = 4;
  }
  for (; L <= M / 2; L <<= 2) {
    const int q = L >> 1, len = 2 * L;
    for (int b = threadIdx.x; b < M / 4; b += blockDim.x) {
      const int j = b % q, base = (b / q) * len + j;
      const cplx a0 = x[base], a1 = x[base + q], a2 = x[base + 2 * q], a3 = x[base + 3 * q];
      const cplx w1 = twiddle(tw, twlen, L, j, sign);
      const cplx w2 = twiddle(tw, twlen, len, j, sign), w2b = twiddle(tw, twlen, len, j + q, sign);
      const cplx t1 = cmul(a1, w1), t3 = cmul(a3, w1);
      const cplx b0 = cadd(a0, t1), b1 = csub(a0, t1), b2 = cadd(a2, t3), b3 = csub(a2, t3);
      const cplx u2 = cmul(b2, w2), u3 = cmul(b3, w2b);
      x[base] = cadd(b0, u2);
      x[base + 2 * q] = csub(b0, u2);
      x[base + q] = cadd(b1, u3);
      x[base + 3 * q] = csub(b1, u3);
    }
    __syncthreads();
  }
}


// e^{i pi k^2 / N}
__device__ __forceinline__ cplx chirp(int k, int N) {
  const long long k2 = ((long long)k * k) % (2LL * N);
  double s, c;
  sincospi((double)k2 / (double)N, &s, &c);
  return {c, s};
}

// e^{2 pi i k / n}
__device__ __forceinline__ cplx unit_root(int k, int n) {
  double s, c;
  sincospi((double)(2 * k) / (double)n, &s, &c);
  return {c, s};
}

__device__ __forceinline__ cplx phase(int m, const DevRing &R, int enabled) {
  if (!enabled || R.phi_num == 0) return {1.0, 0.0};
  const long long den2 = 2LL * R.phi_den;
  const long long num = ((long long)m * R.phi_num) % den2;
  double s, c;
  sincospi((double)num / (double)R.phi_den, &s, &c);
  return {c, s};
}

// Unnormalised length-N DFT with sign (+1 inverse, -1 forward) of the values
// in `buf`.  Power-of-two N: `buf` holds the input in bit-reversed order
// (inverse) or natural order (forward); the result is in natural order
// (inverse) or bit-reversed order (forward).  Other N (Bluestein): `buf` has
// room for M entries, holds the input in natural order in [0, N) and the
// result in natural order in [0, N) for both signs.
__device__ void ring_dft(cplx *buf, const DevRing &R, const RingParams &p, int sign) {
  const int N = R.n / 2;
  if (R.bluestein_m == 0) {
    if (sign > 0) fft_dit(buf, N, p.twiddles, p.twlen, +1);
    else fft_dif(buf, N, p.twiddles, p.twlen, -1);
    return;
  }
  const int M = R.bluestein_m;
  // chirp with w^{-sign}: x_k w_k^{sign}, zero padded
  for (int k = threadIdx.x; k < M; k += blockDim.x) {
    cplx v = {0.0, 0.0};
    if (k < N) {
      cplx w = chirp(k, N);
      if (sign < 0) w = cconj(w);
      v = cmul(buf[k], w);
    }
    buf[k] = v;
  }
  __syncthreads();
  fft_dif(buf, M, p.twiddles, p.twlen, -1);
  // product with the filter spectrum (stored bit-reversed for sign +1; the
  // sign -1 filter is its complex conjugate reflected: F'(p) = conj F(-p))
  const cplx *F = reinterpret_cast<const cplx *>(p.filters) + R.filter;
  const int bits = ilog2(M);
  for (int k = threadIdx.x; k < M; k += blockDim.x) {
    cplx f;
    if (sign > 0) {
      f = F[k];
    } else {
      const unsigned natural = bitrev((unsigned)k, bits);
      const unsigned refl = (M - natural) & (M - 1);
      f = cconj(F[bitrev(refl, bits)]);
    }
    buf[k] = cmul(buf[k], f);
  }
  __syncthreads();
  fft_dit(buf, M, p.twiddles, p.twlen, +1);
  const double inv = 1.0 / (double)M;
  for (int k = threadIdx.x; k < N; k += blockDim.x) {
    cplx w = chirp(k, N);
    if (sign < 0) w = cconj(w);
    buf[k] = cscale(cmul(buf[k], w), inv);
  }
  __syncthreads();
}

__global__ void __launch_bounds__(kRingThreads) k_ring_synthesis(RingParams p) {
  extern __shared__ double smem_d[];
  cplx *sm = reinterpret_cast<cplx *>(smem_d);
  const int kmap = blockIdx.x, r = blockIdx.y;
  const DevRing R = p.rings[r];
  const int n = R.n, N = n / 2;
  const int bits = ilog2(N);
  const bool pow2 = R.bluestein_m == 0;
  cplx *W = sm;            // N + 1
  cplx *buf = sm + N + 1;  // N or M
  const int64_t qstride_m = 2LL * p.ni * p.nvecs;  // q[(2m + odd) * ni * nvecs]
  const int64_t qoff = (int64_t)r * p.nvecs + 2 * kmap;
  const int64_t half = (int64_t)p.ni * p.nvecs;
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
      W[j] = acc;
    }
    __syncthreads();
    for (int k = threadIdx.x; k < N; k += blockDim.x) {
      cplx Wk = W[k], Wc = cconj(W[N - k]);
      if (k == 0) {
        Wk.y = 0.0;
        Wc.y = 0.0;
      }
      const cplx s = cadd(Wk, Wc), d = csub(Wk, Wc);
      const cplx Z = cadd(s, mul_i(cmul(unit_root(k, n), d)));
      buf[pow2 ? bitrev((unsigned)k, bits) : k] = Z;
    }
    __syncthreads();
    ring_dft(buf, R, p, +1);
    const int64_t off = side ? R.off_south : R.off_north;
    for (int s = threadIdx.x; s < N; s += blockDim.x) {
      const cplx z = buf[s];
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
  const int bits = ilog2(N);
  const bool pow2 = R.bluestein_m == 0;
  cplx *F = sm;            // N + 1
  cplx *buf = sm + N + 1;  // N or M
  const int64_t qstride_m = 2LL * p.ni * p.nvecs;
  const int64_t qoff = (int64_t)r * p.nvecs + 2 * kmap;
  const int64_t half = (int64_t)p.ni * p.nvecs;
  for (int side = 0; side < 2; ++side) {
    if (side == 1 && r == 0) break;
    const int64_t off = side ? R.off_south : R.off_north;
    for (int s = threadIdx.x; s < N; s += blockDim.x)
      buf[s] = {p.map_in[(off + 2 * s) * p.nmaps + kmap], p.map_in[(off + 2 * s + 1) * p.nmaps + kmap]};
    __syncthreads();
    ring_dft(buf, R, p, -1);
    // Z in natural order (Bluestein) or bit-reversed (power of two)
    for (int k = threadIdx.x; k <= N; k += blockDim.x) {
      const int k1 = k % N, k2 = (N - k) % N;
      const cplx Zk = buf[pow2 ? bitrev((unsigned)k1, bits) : k1];
      const cplx Zc = cconj(buf[pow2 ? bitrev((unsigned)k2, bits) : k2]);
      const cplx E = cscale(cadd(Zk, Zc), 0.5);
      const cplx D = csub(Zk, Zc);
      const cplx O = {0.5 * D.y, -0.5 * D.x};  // D / (2i)
      F[k] = cadd(E, cmul(cconj(unit_root(k, n)), O));
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

// Plan creation: twiddle table and the Bluestein filter spectra.
__global__ void k_twiddles(double2 *tw, int twlen) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < twlen / 2; k += gridDim.x * blockDim.x) {
    double s, c;
    sincospi((double)(2 * k) / (double)twlen, &s, &c);
    tw[k] = make_double2(c, s);
  }
}

__global__ void __launch_bounds__(kRingThreads) k_bluestein_filters(RingParams p) {
  extern __shared__ double smem_d[];
  cplx *buf = reinterpret_cast<cplx *>(smem_d);
  const DevRing R = p.rings[blockIdx.x];
  if (R.bluestein_m == 0) return;
  const int N = R.n / 2, M = R.bluestein_m;
  // b_k = conj(e^{i pi k^2 / N}) for k in (-N, N), cyclically placed
  for (int k = threadIdx.x; k < M; k += blockDim.x) {
    cplx v = {0.0, 0.0};
    if (k < N) v = cconj(chirp(k, N));
    else if (k > M - N) v = cconj(chirp(M - k, N));
    buf[k] = v;
  }
  __syncthreads();
  fft_dif(buf, M, p.twiddles, p.twlen, -1);
  cplx *F = reinterpret_cast<cplx *>(p.filters_out) + R.filter;
  for (int k = threadIdx.x; k < M; k += blockDim.x) F[k] = buf[k];
}

}  // namespace

size_t ring_smem_bytes(int max_cplx) { return (size_t)max_cplx * sizeof(double) * 2; }

cudaError_t launch_ring_synthesis(const RingParams &prm, cudaStream_t st) {
  const size_t smem = ring_smem_bytes(prm.smem_cplx);
  cudaError_t e = cudaFuncSetAttribute(k_ring_synthesis, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return e;
  dim3 grid(prm.nmaps, prm.ni);
  k_ring_synthesis<<<grid, kRingThreads, smem, st>>>(prm);
  return cudaGetLastError();
}

cudaError_t launch_ring_analysis(const RingParams &prm, cudaStream_t st) {
  const size_t smem = ring_smem_bytes(prm.smem_cplx);
  cudaError_t e = cudaFuncSetAttribute(k_ring_analysis, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return e;
  dim3 grid(prm.nmaps, prm.ni);
  k_ring_analysis<<<grid, kRingThreads, smem, st>>>(prm);
  return cudaGetLastError();
}

cudaError_t launch_ring_setup(const RingParams &prm, double *twiddles, double *filters,
                              cudaStream_t st) {
  k_twiddles<<<64, 256, 0, st>>>(reinterpret_cast<double2 *>(twiddles), prm.twlen);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess || !filters) return e;
  RingParams q = prm;
  q.twiddles = reinterpret_cast<const double2 *>(twiddles);
  q.filters_out = filters;
  const size_t smem = ring_smem_bytes(prm.max_bluestein_m);
  e = cudaFuncSetAttribute(k_bluestein_filters, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  k_bluestein_filters<<<prm.ni, kRingThreads, smem, st>>>(q);
  return cudaGetLastError();
}

}  // namespace wm
