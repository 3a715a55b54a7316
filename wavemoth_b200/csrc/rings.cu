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
// Length-N transforms, in place in shared memory:
//   * N a power of two (every belt ring): radix-2^2 Cooley-Tukey passes.  The
//     inverse reads its input in bit-reversed order (Z is stored there as it
//     is formed) and writes natural order; the forward (decimation in
//     frequency) reads natural order and leaves the spectrum bit-reversed.
//   * any other N (polar rings, n = 4i): Bluestein's chirp-z identity
//     jk = (j^2 + k^2 - (k - j)^2) / 2 turns the DFT into a cyclic convolution
//     of length M = 2^p >= 2N - 1: forward decimation-in-frequency FFT of the
//     chirped input (bit-reversed spectrum), product with the chirp filter's
//     spectrum (precomputed per ring at plan creation, stored bit-reversed),
//     inverse decimation-in-time FFT back to natural order.
// Twiddles come from one table of e^{2 pi i k / TW}, TW the largest power of
// two used; the chirps e^{i pi k^2 / N} and roots e^{2 pi i k / n} of the
// Bluestein rings from a per-ring table; all are computed once, at plan
// creation, with sincospi on exact rationals.
//
// Work decomposition: one CTA per (ring pair, group of G = 2^lg maps), G
// chosen per ring so that the transform buffer (G x N or G x M complex) fits
// 64 KB and three CTAs share an SM.  The G maps are the fastest index of the
// CTA's thread layout: lanes g = 0..G-1 of a warp handle the same bin, pixel
// or butterfly of G maps, so
//   * q rows (16 bytes per map, maps adjacent) are read as G x 16-byte runs,
//   * map pixels (8 bytes per map, maps adjacent) are written as G x 8-byte runs,
//   * twiddles, chirps and phase factors are shared by the G lanes.
// In shared memory element i of map lane g is at slot(i) * G + g with the XOR
// swizzle slot(i) = i ^ ((i >> 3) & 7), a permutation inside each aligned
// group of 8 that spreads the 16-byte accesses of every radix-4 and radix-2
// pass over the 32 banks.
#include <cuda_runtime.h>
#include <stdint.h>

#include "plan.h"
#include "kernels.h"

namespace wm {

namespace {

constexpr int kRingThreads = 256;
constexpr int kPhaseLo = 64;  // e^{i m phi0} = hi[m / 64] * lo[m % 64]

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
__device__ __forceinline__ cplx ld2(const double *p) {
  const double2 v = *reinterpret_cast<const double2 *>(p);
  return {v.x, v.y};
}

__device__ __forceinline__ unsigned bitrev(unsigned k, int bits) {
  return bits ? (__brev(k) >> (32 - bits)) : 0u;
}

__device__ __forceinline__ int ilog2(int v) { return 31 - __clz(v); }

__device__ __forceinline__ int slot(int i) { return i ^ ((i >> 3) & 7); }
__device__ __forceinline__ int at(int i, int g, int lg) { return (slot(i) << lg) + g; }

// tw[k] = e^{2 pi i k / twlen}; returns its conjugate for sign -1
__device__ __forceinline__ cplx twiddle(const double2 *tw, int k, int sign) {
  const double2 t = tw[k];
  return {t.x, sign * t.y};
}

// In-place DIF over the 2^lg interleaved sequences of length M (a power of
// two), natural order in, bit-reversed out.  Consecutive radix-2 stages
// (len, len/2) are fused into one pass (radix 2^2).
__device__ void fft_dif(cplx *x, int M, int lg, const double2 *tw, int twlen, int sign) {
  const int gm = (1 << lg) - 1;
  const int total = (M >> 2) << lg;
  int len = M;
  for (; len >= 4; len >>= 2) {
    const int q = len >> 2, lq = ilog2(q), step = twlen / len;
    for (int t = threadIdx.x; t < total; t += blockDim.x) {
      const int g = t & gm, b = t >> lg;
      const int j = b & (q - 1), base = ((b >> lq) << (lq + 2)) + j;
      const int i0 = at(base, g, lg), i1 = at(base + q, g, lg);
      const int i2 = at(base + 2 * q, g, lg), i3 = at(base + 3 * q, g, lg);
      const cplx a0 = x[i0], a1 = x[i1], a2 = x[i2], a3 = x[i3];
      const cplx w1 = twiddle(tw, j * step, sign), w1b = twiddle(tw, (j + q) * step, sign);
      const cplx w2 = twiddle(tw, 2 * j * step, sign);
      const cplx b0 = cadd(a0, a2), b2 = cmul(csub(a0, a2), w1);
      const cplx b1 = cadd(a1, a3), b3 = cmul(csub(a1, a3), w1b);
      x[i0] = cadd(b0, b1);
      x[i1] = cmul(csub(b0, b1), w2);
      x[i2] = cadd(b2, b3);
      x[i3] = cmul(csub(b2, b3), w2);
    }
    __syncthreads();
  }
  if (len == 2) {
    for (int t = threadIdx.x; t < ((M >> 1) << lg); t += blockDim.x) {
      const int g = t & gm, b = t >> lg;
      const int i0 = at(2 * b, g, lg), i1 = at(2 * b + 1, g, lg);
      const cplx u = x[i0], v = x[i1];
      x[i0] = cadd(u, v);
      x[i1] = csub(u, v);
    }
    __syncthreads();
  }
}

// In-place DIT over 2^lg interleaved sequences: bit-reversed in, natural out;
// stages (L, 2L) fused.
__device__ void fft_dit(cplx *x, int M, int lg, const double2 *tw, int twlen, int sign) {
  const int gm = (1 << lg) - 1;
  const int total = (M >> 2) << lg;
  int L = 2;
  if (ilog2(M) & 1) {
    for (int t = threadIdx.x; t < ((M >> 1) << lg); t += blockDim.x) {
      const int g = t & gm, b = t >> lg;
      const int i0 = at(2 * b, g, lg), i1 = at(2 * b + 1, g, lg);
      const cplx u = x[i0], v = x[i1];
      x[i0] = cadd(u, v);
      x[i1] = csub(u, v);
    }
    __syncthreads();
    L = 4;
  }
  for (; L <= M / 2; L <<= 2) {
    const int q = L >> 1, lq = ilog2(q), len = 2 * L;
    const int s1 = twlen / L, s2 = twlen / len;
    for (int t = threadIdx.x; t < total; t += blockDim.x) {
      const int g = t & gm, b = t >> lg;
      const int j = b & (q - 1), base = ((b >> lq) << (lq + 2)) + j;
      const int i0 = at(base, g, lg), i1 = at(base + q, g, lg);
      const int i2 = at(base + 2 * q, g, lg), i3 = at(base + 3 * q, g, lg);
      const cplx a0 = x[i0], a1 = x[i1], a2 = x[i2], a3 = x[i3];
      const cplx w1 = twiddle(tw, j * s1, sign);
      const cplx w2 = twiddle(tw, j * s2, sign), w2b = twiddle(tw, (j + q) * s2, sign);
      const cplx t1 = cmul(a1, w1), t3 = cmul(a3, w1);
      const cplx b0 = cadd(a0, t1), b1 = csub(a0, t1), b2 = cadd(a2, t3), b3 = csub(a2, t3);
      const cplx u2 = cmul(b2, w2), u3 = cmul(b3, w2b);
      x[i0] = cadd(b0, u2);
      x[i2] = csub(b0, u2);
      x[i1] = cadd(b1, u3);
      x[i3] = csub(b1, u3);
    }
    __syncthreads();
  }
}

// e^{i pi num / den} for an exact rational, reduced modulo 2 first
__device__ __forceinline__ cplx expi_pi(long long num, long long den) {
  const long long r = num % (2 * den);
  double s, c;
  sincospi((double)r / (double)den, &s, &c);
  return {c, s};
}

// e^{2 pi i k / n}, 0 <= k <= n/2
__device__ __forceinline__ cplx ring_root(const RingParams &p, const DevRing &R, int k) {
  const int N = R.n >> 1;
  if (R.bluestein_m == 0) {
    if (k == N) return {-1.0, 0.0};
    const double2 t = p.twiddles[(int64_t)k * (p.twlen / R.n)];
    return {t.x, t.y};
  }
  const double2 t = p.aux[R.aux + N + k];
  return {t.x, t.y};
}

// e^{i pi k^2 / N}, k < N (Bluestein rings)
__device__ __forceinline__ cplx ring_chirp(const RingParams &p, const DevRing &R, int k) {
  const double2 t = p.aux[R.aux + k];
  return {t.x, t.y};
}

// Phase factor tables of one ring: lo[b] = e^{i b phi0}, hi[a] = e^{i 64 a phi0}
// (all ones when phase shifting is off or phi0 = 0).
__device__ void phase_tables(cplx *lo, cplx *hi, const RingParams &p, const DevRing &R) {
  const bool on = p.phase_shifts && R.phi_num != 0;
  for (int k = threadIdx.x; k < kPhaseLo + p.nphase_hi; k += blockDim.x) {
    const long long m = k < kPhaseLo ? k : (long long)(k - kPhaseLo) * kPhaseLo;
    const cplx v = on ? expi_pi(m * R.phi_num, R.phi_den) : cplx{1.0, 0.0};
    if (k < kPhaseLo) lo[k] = v;
    else hi[k - kPhaseLo] = v;
  }
}

__device__ __forceinline__ cplx phase_at(const cplx *lo, const cplx *hi, int m) {
  return cmul(hi[m >> 6], lo[m & (kPhaseLo - 1)]);
}

struct RingCta {
  DevRing R;
  int ring, map0, lg, nm;  // nm: maps of the group that exist
  int n, N, M, bits, bitsM;
  bool pow2;
};

__device__ __forceinline__ RingCta ring_cta(const RingParams &p, int task) {
  RingCta c;
  const DevRingTask T = p.tasks[task];
  c.R = p.rings[T.ring];
  c.ring = T.ring;
  c.map0 = T.map0;
  c.lg = T.lg;
  c.nm = min(1 << T.lg, p.nmaps - T.map0);
  c.n = c.R.n;
  c.N = c.n >> 1;
  c.pow2 = c.R.bluestein_m == 0;
  c.M = c.pow2 ? c.N : c.R.bluestein_m;
  c.bits = ilog2(c.N);
  c.bitsM = ilog2(c.M);
  return c;
}

// Cyclic convolution step of Bluestein's method on the chirped, zero-padded
// buffer (natural order in, natural order out).
__device__ void bluestein_convolve(cplx *buf, const RingCta &c, const RingParams &p, int sign) {
  const int gm = (1 << c.lg) - 1, M = c.M;
  fft_dif(buf, M, c.lg, p.twiddles, p.twlen, -1);
  // filter spectrum, stored bit-reversed for sign +1; the sign -1 filter is
  // its reflection F'(k) = F(-k), conjugated
  const cplx *F = reinterpret_cast<const cplx *>(p.filters) + c.R.filter;
  for (int t = threadIdx.x; t < (M << c.lg); t += blockDim.x) {
    const int g = t & gm, k = t >> c.lg;
    cplx f;
    if (sign > 0) {
      f = F[k];
    } else {
      const unsigned natural = bitrev((unsigned)k, c.bitsM);
      const unsigned refl = (M - natural) & (M - 1);
      f = cconj(F[bitrev(refl, c.bitsM)]);
    }
    const int i = at(k, g, c.lg);
    buf[i] = cmul(buf[i], f);
  }
  __syncthreads();
  fft_dit(buf, M, c.lg, p.twiddles, p.twlen, +1);
}

// W[j] of one map (q row pointer `qg` at ring r, map g), aliasing sum in increasing m
__device__ __forceinline__ cplx alias_sum(const double *qg, int j, int n, int mmax,
                                          int64_t qstride, int64_t half, double sgn,
                                          const cplx *plo, const cplx *phi) {
  cplx acc = {0.0, 0.0};
  for (int base = 0;; base += n) {
    const int m1 = base + j;
    if (m1 > mmax) break;
    {
      const cplx e = ld2(qg + m1 * qstride), o = ld2(qg + m1 * qstride + half);
      const cplx t = {e.x + sgn * o.x, e.y + sgn * o.y};
      acc = cadd(acc, cmul(t, phase_at(plo, phi, m1)));
    }
    const int m2 = base + n - j;
    if (m2 <= mmax) {
      const cplx e = ld2(qg + m2 * qstride), o = ld2(qg + m2 * qstride + half);
      const cplx t = {e.x + sgn * o.x, e.y + sgn * o.y};
      acc = cadd(acc, cconj(cmul(t, phase_at(plo, phi, m2))));
    }
  }
  return acc;
}

__global__ void __launch_bounds__(kRingThreads, 3) k_ring_synthesis(RingParams p, int task0) {
  extern __shared__ double smem_d[];
  const RingCta c = ring_cta(p, task0 + blockIdx.x);
  const int lg = c.lg, gm = (1 << lg) - 1, n = c.n, N = c.N;
  cplx *buf = reinterpret_cast<cplx *>(smem_d);
  cplx *plo = buf + ((int64_t)c.M << lg);
  cplx *phi = plo + kPhaseLo;
  phase_tables(plo, phi, p, c.R);
  __syncthreads();
  const int64_t half = (int64_t)p.ni * p.nvecs, qstride = 2 * half;
  const double *qbase = p.q + (int64_t)c.ring * p.nvecs + 2 * c.map0;
  for (int side = 0; side < 2; ++side) {
    if (side == 1 && c.ring == 0) break;  // the equator is written once
    const double sgn = side ? -1.0 : 1.0;
    // Z[k] and Z[N - k] from W[k] and W[N - k]
    const int npairs = (N >> 1) + 1;
    for (int t = threadIdx.x; t < (npairs << lg); t += blockDim.x) {
      const int g = t & gm, kk = t >> lg, kr = N - kk;
      cplx Wa = {0.0, 0.0}, Wb = {0.0, 0.0};  // W[kk], W[N - kk]
      if (g < c.nm) {
        const double *qg = qbase + 2 * g;
        Wa = alias_sum(qg, kk, n, p.mmax, qstride, half, sgn, plo, phi);
        Wb = kr == kk ? Wa : alias_sum(qg, kr, n, p.mmax, qstride, half, sgn, plo, phi);
      }
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int k = e ? kr : kk;
        if (e && (kr == kk || kr == N)) break;
        cplx Wk = e ? Wb : Wa, Wc = cconj(e ? Wa : Wb);
        if (k == 0) {
          Wk.y = 0.0;
          Wc.y = 0.0;
        }
        const cplx s = cadd(Wk, Wc), d = csub(Wk, Wc);
        cplx Z = cadd(s, mul_i(cmul(ring_root(p, c.R, k), d)));
        if (c.pow2) {
          buf[at((int)bitrev((unsigned)k, c.bits), g, lg)] = Z;
        } else {
          buf[at(k, g, lg)] = cmul(Z, ring_chirp(p, c.R, k));
        }
      }
    }
    if (!c.pow2)
      for (int t = threadIdx.x; t < ((c.M - N) << lg); t += blockDim.x)
        buf[at(N + (t >> lg), t & gm, lg)] = {0.0, 0.0};
    __syncthreads();
    if (c.pow2) fft_dit(buf, N, lg, p.twiddles, p.twlen, +1);
    else bluestein_convolve(buf, c, p, +1);
    const int64_t off = side ? c.R.off_south : c.R.off_north;
    const double inv = c.pow2 ? 1.0 : 1.0 / (double)c.M;
    double *out = p.map + off * p.nmaps + c.map0;
    for (int t = threadIdx.x; t < (n << lg); t += blockDim.x) {
      const int g = t & gm, pix = t >> lg, s = pix >> 1;
      if (g >= c.nm) continue;
      cplx z = buf[at(s, g, lg)];
      if (!c.pow2) z = cscale(cmul(z, ring_chirp(p, c.R, s)), inv);
      out[(int64_t)pix * p.nmaps + g] = (pix & 1) ? z.y : z.x;
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kRingThreads, 3) k_ring_analysis(RingParams p, int task0) {
  extern __shared__ double smem_d[];
  const RingCta c = ring_cta(p, task0 + blockIdx.x);
  const int lg = c.lg, gm = (1 << lg) - 1, n = c.n, N = c.N;
  cplx *buf = reinterpret_cast<cplx *>(smem_d);
  cplx *plo = buf + ((int64_t)c.M << lg);
  cplx *phi = plo + kPhaseLo;
  phase_tables(plo, phi, p, c.R);
  const int64_t half = (int64_t)p.ni * p.nvecs, qstride = 2 * half;
  double *qbase = p.q_out + (int64_t)c.ring * p.nvecs + 2 * c.map0;
  const double inv = c.pow2 ? 1.0 : 1.0 / (double)c.M;
  for (int side = 0; side < 2; ++side) {
    if (side == 1 && c.ring == 0) break;
    const int64_t off = side ? c.R.off_south : c.R.off_north;
    const double *in = p.map_in + off * p.nmaps + c.map0;
    for (int t = threadIdx.x; t < (N << lg); t += blockDim.x) {
      const int g = t & gm, s = t >> lg;
      cplx z = {0.0, 0.0};
      if (g < c.nm) z = {in[(int64_t)(2 * s) * p.nmaps + g], in[(int64_t)(2 * s + 1) * p.nmaps + g]};
      if (!c.pow2) z = cmul(z, cconj(ring_chirp(p, c.R, s)));
      buf[at(s, g, lg)] = z;
    }
    if (!c.pow2)
      for (int t = threadIdx.x; t < ((c.M - N) << lg); t += blockDim.x)
        buf[at(N + (t >> lg), t & gm, lg)] = {0.0, 0.0};
    __syncthreads();
    if (c.pow2) fft_dif(buf, N, lg, p.twiddles, p.twlen, -1);
    else bluestein_convolve(buf, c, p, -1);
    // fold the spectrum F[k] (k <= N) into q~: g_m = F[m mod n] or its mirror
    for (int t = threadIdx.x; t < ((p.mmax + 1) << lg); t += blockDim.x) {
      const int g = t & gm, m = t >> lg;
      if (g >= c.nm) continue;
      const int jm = m % n;
      const bool mirror = jm > N;
      const int k = mirror ? n - jm : jm;
      const int k1 = k == N ? 0 : k, k2 = k == 0 ? 0 : N - k;
      cplx Zk, Zc;
      if (c.pow2) {
        Zk = buf[at((int)bitrev((unsigned)k1, c.bits), g, lg)];
        Zc = buf[at((int)bitrev((unsigned)k2, c.bits), g, lg)];
      } else {
        Zk = cscale(cmul(buf[at(k1, g, lg)], cconj(ring_chirp(p, c.R, k1))), inv);
        Zc = cscale(cmul(buf[at(k2, g, lg)], cconj(ring_chirp(p, c.R, k2))), inv);
      }
      Zc = cconj(Zc);
      const cplx E = cscale(cadd(Zk, Zc), 0.5);
      const cplx D = csub(Zk, Zc);
      const cplx O = {0.5 * D.y, -0.5 * D.x};  // D / (2i)
      cplx F = cadd(E, cmul(cconj(ring_root(p, c.R, k)), O));
      if (mirror) F = cconj(F);
      const cplx gv = cscale(cmul(F, cconj(phase_at(plo, phi, m))), p.scale);
      double *qe = qbase + m * qstride + 2 * g;
      double *qo = qe + half;
      if (side == 0) {
        *reinterpret_cast<double2 *>(qe) = make_double2(gv.x, gv.y);
        *reinterpret_cast<double2 *>(qo) = make_double2(gv.x, gv.y);
      } else {
        const cplx e = ld2(qe), o = ld2(qo);
        *reinterpret_cast<double2 *>(qe) = make_double2(e.x + gv.x, e.y + gv.y);
        *reinterpret_cast<double2 *>(qo) = make_double2(o.x - gv.x, o.y - gv.y);
      }
    }
    __syncthreads();
  }
}

// Plan creation: twiddle table, Bluestein chirp/root tables and filter spectra.
__global__ void k_twiddles(double2 *tw, int twlen) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < twlen / 2; k += gridDim.x * blockDim.x) {
    const cplx v = expi_pi(2LL * k, twlen);
    tw[k] = make_double2(v.x, v.y);
  }
}

__global__ void k_ring_aux(RingParams p) {
  const DevRing R = p.rings[blockIdx.x];
  if (R.bluestein_m == 0) return;
  const int N = R.n / 2;
  double2 *aux = reinterpret_cast<double2 *>(p.aux_out) + R.aux;
  for (int k = threadIdx.x; k < N; k += blockDim.x) {
    const cplx v = expi_pi((long long)k * k, N);  // e^{i pi k^2 / N}
    aux[k] = make_double2(v.x, v.y);
  }
  for (int k = threadIdx.x; k <= N; k += blockDim.x) {
    const cplx v = expi_pi(2LL * k, R.n);  // e^{2 pi i k / n}
    aux[N + k] = make_double2(v.x, v.y);
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
    if (k < N) v = cconj(expi_pi((long long)k * k, N));
    else if (k > M - N) v = cconj(expi_pi((long long)(M - k) * (M - k), N));
    buf[at(k, 0, 0)] = v;
  }
  __syncthreads();
  fft_dif(buf, M, 0, p.twiddles, p.twlen, -1);
  cplx *F = reinterpret_cast<cplx *>(p.filters_out) + R.filter;
  for (int k = threadIdx.x; k < M; k += blockDim.x) F[k] = buf[at(k, 0, 0)];
}

template <class K>
cudaError_t launch_classes(K kernel, const RingParams &prm, cudaStream_t st) {
  const int smem_max = prm.smem0 > prm.smem1 ? prm.smem0 : prm.smem1;
  cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_max);
  if (e != cudaSuccess) return e;
  if (prm.ntasks0 > 0) {
    kernel<<<prm.ntasks0, kRingThreads, prm.smem0, st>>>(prm, 0);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  if (prm.ntasks1 > 0) {
    kernel<<<prm.ntasks1, kRingThreads, prm.smem1, st>>>(prm, prm.ntasks0);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  return cudaSuccess;
}

}  // namespace

int32_t ring_cta_smem(int64_t buffer_cplx, int32_t nphase_hi) {
  return (int32_t)((buffer_cplx + kPhaseLo + nphase_hi) * 2 * sizeof(double));
}

cudaError_t launch_ring_synthesis(const RingParams &prm, cudaStream_t st) {
  return launch_classes(k_ring_synthesis, prm, st);
}

cudaError_t launch_ring_analysis(const RingParams &prm, cudaStream_t st) {
  return launch_classes(k_ring_analysis, prm, st);
}

cudaError_t launch_ring_setup(const RingParams &prm, double *twiddles, double *filters, double *aux,
                              cudaStream_t st) {
  k_twiddles<<<64, 256, 0, st>>>(reinterpret_cast<double2 *>(twiddles), prm.twlen);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess || !filters) return e;
  RingParams q = prm;
  q.twiddles = reinterpret_cast<const double2 *>(twiddles);
  q.filters_out = filters;
  q.aux_out = aux;
  k_ring_aux<<<prm.ni, 256, 0, st>>>(q);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  const int smem = prm.max_bluestein_m * 2 * (int)sizeof(double);
  e = cudaFuncSetAttribute(k_bluestein_filters, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return e;
  k_bluestein_filters<<<prm.ni, kRingThreads, smem, st>>>(q);
  return cudaGetLastError();
}

}  // namespace wm
