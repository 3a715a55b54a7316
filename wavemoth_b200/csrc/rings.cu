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
// Length-N transforms, in place in shared memory, as passes of radix 16 (and
// one last decimation-in-frequency pass of radix 2, 4 or 8 when log2 of the
// length is not a multiple of 4); a pass loads 16 points per butterfly into
// registers and runs four radix-2 stages there.  The first radix-16 pass of
// a decimation in frequency leaves 16 independent blocks per lane; each of
// the CTA's 16 warps owns one and runs the later passes (the earlier ones of
// a decimation in time) on it alone, with warp barriers in place of CTA
// barriers:
//   * N a power of two (every belt ring): synthesis by decimation in
//     frequency (natural order in, bit-reversed out), analysis by decimation
//     in time (bit-reversed in, natural out).  Z is formed in natural order
//     as W is gathered from q, the last synthesis pass writes the ring
//     pixels from its registers and the first analysis pass loads them.
//   * any other N (polar rings, n = 4i): Bluestein's chirp-z identity
//     jk = (j^2 + k^2 - (k - j)^2) / 2 turns the DFT into a cyclic convolution
//     of length M = 2^p >= 2N - 1: DIF of the chirped, zero-padded input, the
//     product with the chirp filter's spectrum (precomputed per ring, stored
//     in the DIF output order) and DIT back; the last DIF pass, the product
//     and the first DIT pass share one register pass.
// Within a radix-16 pass the twiddles of radix-2 stage s at offset
// j + m (len / 16) factor as w_{len / 2^s}^j (one table lookup per stage,
// all four issued before the butterfly's points are loaded; every length is
// a power of two, so the index is a shift of j) times a 16th root of unity
// fixed at compile time.  Twiddles come from one table of e^{2 pi i k / TW},
// TW the largest power of two used; chirps e^{i pi k^2 / N} and roots
// e^{2 pi i k / n} of the Bluestein rings from a per-ring table; all computed
// at plan creation with sincospi on exact rationals.
//
// Work decomposition: one CTA of 512 threads per (ring pair, group of G = 2^lg
// maps) with a 128 KB transform buffer (8192 complex, 16 points per thread).
// Both hemispheres of the pair share the CTA when 2 G x N (or 2 G x M) fits
// the buffer: lanes are (side, map), so synthesis reads every q element once
// and analysis writes every q~ element once; longer transforms (nside 2048)
// run one hemisphere at a time.  Lanes are the fastest index of the thread
// layout: lanes of a warp handle the same bin, pixel or butterfly of
// different maps, so q rows and map pixels are read and written as G-map runs
// and twiddles, chirps and phases are shared.
// In shared memory element i of lane g is at slot(i) * lanes + g with the XOR
// swizzle slot(i) = i ^ ((i >> 4) & 15), a permutation inside each aligned
// group of 16 that makes the 16-byte accesses of every pass of radix 2..16
// conflict-free for 1, 2, 4, 8 and 16 lanes.
#include <cuda_runtime.h>

#include <algorithm>
#include <stdint.h>

#include "plan.h"
#include "kernels.h"

namespace wm {

namespace {

constexpr int kRadixLog = 4;           // largest pass radix 2^kRadixLog
constexpr int kRingThreads = 512;      // 16 points per thread of a kRingBufferCplx buffer
constexpr int kRingWarps = kRingThreads / 32;
static_assert(kRingWarps == 16, "warp-local passes give each of 16 warps the blocks of a radix-16 pass");
constexpr int kPhaseLo = kRingPhaseLo;  // e^{i m phi0} = hi[m / 64] * lo[m % 64]

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
__device__ __forceinline__ void st2(double *p, double x, double y) {
  *reinterpret_cast<double2 *>(p) = make_double2(x, y);
}

__device__ __forceinline__ unsigned bitrev(unsigned k, int bits) {
  return bits ? (__brev(k) >> (32 - bits)) : 0u;
}

__device__ __forceinline__ int ilog2(int v) { return 31 - __clz(v); }

__device__ __forceinline__ int slot(int i) { return i ^ ((i >> 4) & 15); }
__device__ __forceinline__ int at(int i, int g, int lg) { return (slot(i) << lg) + g; }

// tw[k] = e^{2 pi i k / twlen}; its conjugate for SIGN = -1
template <int SIGN>
__device__ __forceinline__ cplx twiddle(const double2 *tw, int k) {
  const double2 t = tw[k];
  return {t.x, SIGN * t.y};
}

// a e^{SIGN 2 pi i k / 16} for a k known after unrolling
template <int SIGN>
__device__ __forceinline__ cplx mul_root16(cplx a, int k) {
  // cos and sin of 2 pi k / 16, k = 0..3 (the rest by symmetry)
  constexpr double c1 = 0.92387953251128675613, s1 = 0.38268343236508977173;
  constexpr double h = 0.70710678118654752440;
  k &= 15;
  if (k == 0) return a;
  if (k == 4) return SIGN > 0 ? cplx{-a.y, a.x} : cplx{a.y, -a.x};
  if (k == 8) return {-a.x, -a.y};
  if (k == 12) return SIGN > 0 ? cplx{a.y, -a.x} : cplx{-a.y, a.x};
  double c, s;
  switch (k & 3) {
    case 1: c = c1; s = s1; break;
    case 2: c = h; s = h; break;
    default: c = s1; s = c1; break;
  }
  // quadrant of k: rotate (c, s) by multiples of pi/2
  const int qd = k >> 2;
  double cc = c, ss = s;
  if (qd == 1) { cc = -s; ss = c; }
  else if (qd == 2) { cc = -c; ss = -s; }
  else if (qd == 3) { cc = s; ss = -c; }
  return cmul(a, cplx{cc, SIGN * ss});
}

template <int R>
struct Log2;
template <> struct Log2<2> { static constexpr int v = 1; };
template <> struct Log2<4> { static constexpr int v = 2; };
template <> struct Log2<8> { static constexpr int v = 3; };
template <> struct Log2<16> { static constexpr int v = 4; };

// Stage twiddles of a radix-R butterfly at offset j of a block of length
// 2^lglen, fetched before the butterfly's points: DIF stage s uses
// w_{len / 2^s}^j, DIT stage s uses w_{2^(s+1) len / R}^j.  All lengths are
// powers of two, so the table index is a shift of j.
template <int R, int SIGN, bool DIF>
__device__ __forceinline__ void stage_twiddles(cplx (&A)[Log2<R>::v], int j, int lglen, const double2 *tw,
                                               int lgtw) {
#pragma unroll
  for (int s = 0; s < Log2<R>::v; ++s) {
    const int sh = DIF ? lgtw - lglen + s : lgtw - lglen + Log2<R>::v - (s + 1);
    A[s] = twiddle<SIGN>(tw, j << sh);
  }
}

// Radix-R decimation-in-frequency butterfly of R points in registers:
// log2 R radix-2 stages, stage s multiplied by A[s] and a 16th root.
template <int R, int SIGN>
__device__ __forceinline__ void dif_regs(cplx (&x)[R], const cplx (&A)[Log2<R>::v]) {
#pragma unroll
  for (int s = 0; s < Log2<R>::v; ++s) {
    const int h = R >> (s + 1);
#pragma unroll
    for (int i = 0; i < R / 2; ++i) {
      const int lo = (i / h) * 2 * h + (i % h), hi = lo + h, m = i % h;
      const cplx u = x[lo], v = x[hi];
      x[lo] = cadd(u, v);
      x[hi] = mul_root16<SIGN>(cmul(csub(u, v), A[s]), (m << s) * (16 / R));
    }
  }
}

// Radix-R decimation-in-time butterfly of R points in registers.
template <int R, int SIGN>
__device__ __forceinline__ void dit_regs(cplx (&x)[R], const cplx (&A)[Log2<R>::v]) {
#pragma unroll
  for (int s = 0; s < Log2<R>::v; ++s) {
    const int h = 1 << s;
#pragma unroll
    for (int i = 0; i < R / 2; ++i) {
      const int lo = (i / h) * 2 * h + (i % h), hi = lo + h, m = i % h;
      const cplx u = x[lo];
      const cplx t = mul_root16<SIGN>(cmul(x[hi], A[s]), m << (4 - (s + 1)));
      x[lo] = cadd(u, t);
      x[hi] = csub(u, t);
    }
  }
}

}  // namespace
}  // namespace wm

namespace wm {
namespace {

// Shared arguments of the passes of one CTA: the twiddle table (2^lgtw
// entries), the transform length M and the log2 of the lanes.
struct FftCtx {
  const double2 *tw;
  int lgtw;
  int M;
  int lg;
};

// Butterflies of a pass, `body(b, g)` for butterfly b (per lane) of lane g.
// wl == 0: all the CTA's threads over all butterflies, then a CTA barrier.
// wl > 0: warp w alone runs the butterflies inside its own blocks of 2^wl
// points of every lane, then a warp barrier -- for the passes after the
// first radix-16 pass of a decimation in frequency (and before the last of
// a decimation in time), whose blocks nest in those the warp owns, so that
// warps run these passes without waiting for one another.
template <int LR, class BodyF>
__device__ __forceinline__ void for_butterflies(const FftCtx &f, int wl, BodyF body) {
  const int gm = (1 << f.lg) - 1;
  if (wl == 0) {
    const int nbf = (f.M >> LR) << f.lg;
    for (int t = threadIdx.x; t < nbf; t += blockDim.x) body(t >> f.lg, t & gm);
    __syncthreads();
  } else {
    // warp w owns the blocks [w k, (w + 1) k): nblk >= 16 blocks (a power of
    // two) over the CTA's 16 warps; its lanes run over (block, butterfly)
    const int k = (f.M >> wl) / kRingWarps, warp = threadIdx.x >> 5;
    const int lp = wl - LR + f.lg;  // log2 of the butterflies of one block, all lanes
    for (int i = threadIdx.x & 31; i < (k << lp); i += 32) {
      const int B = warp * k + (i >> lp), u = i & ((1 << lp) - 1);
      body((B << (wl - LR)) + (u >> f.lg), u & gm);
    }
    __syncwarp();
  }
}

// One in-place pass of radix R over the 2^lg interleaved sequences of length
// M: butterfly b of lane g takes the points base + i q (q = len / R, len =
// 2^lglen) of its block, through `load(index, g)` and `store(index, g, value)`.
template <int R, int SIGN, bool DIF, class LoadF, class StoreF>
__device__ __forceinline__ void fft_pass(const FftCtx &f, int lglen, int wl, LoadF load, StoreF store) {
  constexpr int LR = Log2<R>::v;
  const int lq = lglen - LR;
  for_butterflies<LR>(f, wl, [&](int b, int g) {
    const int j = b & ((1 << lq) - 1), base = ((b >> lq) << lglen) + j;
    cplx A[LR];
    stage_twiddles<R, SIGN, DIF>(A, j, lglen, f.tw, f.lgtw);
    cplx x[R];
#pragma unroll
    for (int i = 0; i < R; ++i) x[i] = load(base + (i << lq), g);
    if (DIF) dif_regs<R, SIGN>(x, A);
    else dit_regs<R, SIGN>(x, A);
#pragma unroll
    for (int i = 0; i < R; ++i) store(base + (i << lq), g, x[i]);
  });
}

template <int SIGN, bool DIF, class LoadF, class StoreF>
__device__ __forceinline__ void fft_pass_r(const FftCtx &f, int R, int lglen, int wl, LoadF load, StoreF store) {
  switch (R) {
    case 2: fft_pass<2, SIGN, DIF>(f, lglen, wl, load, store); break;
    case 4: fft_pass<4, SIGN, DIF>(f, lglen, wl, load, store); break;
    case 8:
      if (kRadixLog > 3) {
        fft_pass<8, SIGN, DIF>(f, lglen, wl, load, store);
        break;
      }
      [[fallthrough]];
    default: fft_pass<(1 << kRadixLog), SIGN, DIF>(f, lglen, wl, load, store); break;
  }
}

// Middle of Bluestein's convolution on blocks of R points (R = the last DIF
// radix = the first DIT radix): forward DIF stages, the product with the
// filter spectrum (stored in DIF output order; the sign -1 filter is its
// reflection F'(k) = conj F(-k)), inverse DIT stages.  Block offset 0: every
// stage twiddle is 1.
template <int R, class LoadF, class StoreF>
__device__ __forceinline__ void bluestein_mid_r(const FftCtx &f, const cplx *F, int fsign, int wl, LoadF load,
                                                StoreF store) {
  const int bitsM = ilog2(f.M);
  cplx one[Log2<R>::v];
#pragma unroll
  for (int s = 0; s < Log2<R>::v; ++s) one[s] = {1.0, 0.0};
  for_butterflies<Log2<R>::v>(f, wl, [&](int b, int g) {
    const int base = b * R;
    cplx x[R];
#pragma unroll
    for (int i = 0; i < R; ++i) x[i] = load(base + i, g);
    dif_regs<R, -1>(x, one);
#pragma unroll
    for (int i = 0; i < R; ++i) {
      const int k = base + i;
      cplx fk;
      if (fsign > 0) {
        fk = F[k];
      } else {
        const unsigned natural = bitrev((unsigned)k, bitsM);
        const unsigned refl = (f.M - natural) & (f.M - 1);
        fk = cconj(F[bitrev(refl, bitsM)]);
      }
      x[i] = cmul(x[i], fk);
    }
    dit_regs<R, 1>(x, one);
#pragma unroll
    for (int i = 0; i < R; ++i) store(base + i, g, x[i]);
  });
}

template <class LoadF, class StoreF>
__device__ __forceinline__ void bluestein_mid(const FftCtx &f, int R, const cplx *F, int fsign, int wl, LoadF load,
                                              StoreF store) {
  switch (R) {
    case 2: bluestein_mid_r<2>(f, F, fsign, wl, load, store); break;
    case 4: bluestein_mid_r<4>(f, F, fsign, wl, load, store); break;
    case 8:
      if (kRadixLog > 3) {
        bluestein_mid_r<8>(f, F, fsign, wl, load, store);
        break;
      }
      [[fallthrough]];
    default: bluestein_mid_r<(1 << kRadixLog)>(f, F, fsign, wl, load, store); break;
  }
}

// Pass radices of a length-M transform in DIF order: the radix-16 passes
// and one pass of radix 2^(log2 M mod 4) (if above 1), first or last.  DIT
// runs them in reverse order.  Once the passes before p have cut every
// lane into at least 16 blocks (one or more per warp of the CTA), pass p and
// the later DIF passes (the earlier DIT passes) run warp-local on the blocks
// of pass p0 (for_butterflies).  Computed per pass (no per-thread arrays,
// which would live in local memory).
template <bool kSmallFirst>
struct Radices {
  int lgM;  // log2 M
  int r0;   // log2 M mod 4: log2 of the small radix, 0 if none
  int n;    // number of passes
  // radix of DIF pass p
  __device__ __forceinline__ int r(int p) const {
    return (r0 && p == (kSmallFirst ? 0 : n - 1)) ? 1 << r0 : 1 << kRadixLog;
  }
  // log2 of the block length of DIF pass p (the DIT pass mirroring it has the same)
  __device__ __forceinline__ int lgl(int p) const {
    return lgM - kRadixLog * p + ((kSmallFirst && r0 && p > 0) ? kRadixLog - r0 : 0);
  }
  // first warp-local DIF pass: the first after a radix-16 pass
  __device__ __forceinline__ int p0() const { return (kSmallFirst && r0) ? 2 : 1; }
  // log2 of the per-lane block a warp owns in pass p (0: the whole CTA runs the pass)
  __device__ __forceinline__ int wl(int p) const { return (p >= p0() && p < n) ? lgl(p0()) : 0; }
};

template <bool kSmallFirst>
__device__ __forceinline__ Radices<kSmallFirst> radices(int M) {
  Radices<kSmallFirst> s;
  s.lgM = ilog2(M);
  s.r0 = s.lgM % kRadixLog;
  s.n = s.lgM / kRadixLog + (s.r0 ? 1 : 0);
  return s;
}

}  // namespace
}  // namespace wm

namespace wm {
namespace {

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
    const double2 t = p.twiddles[k << (ilog2(p.twlen) - ilog2(R.n))];
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
// (all ones when phase shifting is off or phi0 = 0), copied into shared
// memory from the per-ring table made at plan creation (k_ring_phases).
__device__ void phase_tables(cplx *lo, cplx *hi, const RingParams &p, int ring) {
  const bool on = p.phase_shifts != 0;
  const double2 *src = p.phases + (int64_t)ring * (kPhaseLo + p.nphase_hi);
  for (int k = threadIdx.x; k < kPhaseLo + p.nphase_hi; k += blockDim.x) {
    const double2 t = on ? src[k] : make_double2(1.0, 0.0);
    if (k < kPhaseLo) lo[k] = {t.x, t.y};
    else hi[k - kPhaseLo] = {t.x, t.y};
  }
}

__device__ __forceinline__ cplx phase_at(const cplx *lo, const cplx *hi, int m) {
  return cmul(hi[m >> 6], lo[m & (kPhaseLo - 1)]);
}

struct RingCta {
  DevRing R;
  int ring, map0;
  int lgm;   // log2 of the maps per CTA
  int two;   // 1: both hemispheres in the CTA (lane g = side * 2^lgm + map)
  int lg;    // log2 of the lanes: lgm + two
  int nm;    // maps of the group that exist
  int n, N, M, bits;
  bool pow2;
};

__device__ __forceinline__ RingCta ring_cta(const RingParams &p, int task) {
  RingCta c;
  const DevRingTask T = p.tasks[task];
  c.R = p.rings[T.ring];
  c.ring = T.ring;
  c.map0 = T.map0;
  c.lgm = T.lg;
  c.two = T.pad;
  c.lg = T.lg + T.pad;
  c.nm = min(1 << T.lg, p.nmaps - T.map0);
  c.n = c.R.n;
  c.N = c.n >> 1;
  c.pow2 = c.R.bluestein_m == 0;
  c.M = c.pow2 ? c.N : c.R.bluestein_m;
  c.bits = ilog2(c.N);
  return c;
}

// Lane g of a CTA: its map (within the group) and hemisphere (0 north, 1
// south); `side` is the hemisphere of a CTA that runs them one at a time.
__device__ __forceinline__ int lane_map(const RingCta &c, int g) { return g & ((1 << c.lgm) - 1); }
__device__ __forceinline__ int lane_side(const RingCta &c, int g, int side) { return c.two ? g >> c.lgm : side; }
__device__ __forceinline__ bool lane_live(const RingCta &c, int g, int side) {
  return lane_map(c, g) < c.nm && !(lane_side(c, g, side) == 1 && c.ring == 0);
}

// q values (even part a, odd part b) of the first term of the aliasing sums
// of bin j, m = j (zero when j > mmax).  Loaded one item ahead of the sums,
// so that a thread's next q loads are in flight while it sums.
__device__ __forceinline__ void first_term(const double *qg, int j, int mmax, int64_t qstride, int64_t half,
                                           bool live, cplx &a, cplx &b) {
  if (live && j <= mmax) {
    a = ld2(qg + j * qstride);
    b = ld2(qg + j * qstride + half);
  } else {
    a = {0.0, 0.0};
    b = {0.0, 0.0};
  }
}

// Even and odd partial sums of W[j] of one map (q row pointer `qg` at ring r,
// map g; a0, b0 the q values at m = j): W = A + B on the northern ring,
// A - B on the southern one; the aliasing sum runs in increasing m.
__device__ __forceinline__ void alias_sums(const double *qg, int j, int n, int mmax, int64_t qstride,
                                           int64_t half, const cplx *plo, const cplx *phi, cplx a0, cplx b0,
                                           cplx &A, cplx &B) {
  A = {0.0, 0.0};
  B = {0.0, 0.0};
  for (int base = 0;; base += n) {
    const int m1 = base + j;
    if (m1 > mmax) break;
    {
      const cplx ph = phase_at(plo, phi, m1);
      const cplx a = base ? ld2(qg + m1 * qstride) : a0, b = base ? ld2(qg + m1 * qstride + half) : b0;
      A = cadd(A, cmul(a, ph));
      B = cadd(B, cmul(b, ph));
    }
    const int m2 = base + n - j;
    if (m2 <= mmax) {
      const cplx ph = phase_at(plo, phi, m2);
      A = cadd(A, cconj(cmul(ld2(qg + m2 * qstride), ph)));
      B = cadd(B, cconj(cmul(ld2(qg + m2 * qstride + half), ph)));
    }
  }
}

__global__ void __launch_bounds__(kRingThreads, 1) k_ring_synthesis(RingParams p) {
  extern __shared__ double smem_d[];
  const RingCta c = ring_cta(p, blockIdx.x);
  const int lg = c.lg, gm = (1 << lg) - 1, n = c.n, N = c.N, M = c.M;
  cplx *buf = reinterpret_cast<cplx *>(smem_d);
  cplx *plo = buf + ((int64_t)M << lg);
  cplx *phi = plo + kPhaseLo;
  phase_tables(plo, phi, p, c.ring);
  __syncthreads();
  // q rows are ring-major: (m, parity) of ring r at row (r (mmax + 1) + m) 2 + parity
  const int64_t half = p.nvecs, qstride = 2 * half;
  const double *qbase = p.q + (int64_t)c.ring * (p.mmax + 1) * qstride + 2 * c.map0;
  // the aliasing sums stop at the ring's m limit (null: every m)
  const int mlim = p.ring_mend ? p.ring_mend[c.ring] - 1 : p.mmax;
  const auto rs = radices<false>(M);
  const FftCtx fx{p.twiddles, ilog2(p.twlen), M, lg};
  const cplx *F = reinterpret_cast<const cplx *>(p.filters) + c.R.filter;
  const double inv = (c.pow2 ? 1.0 : 1.0 / (double)M) * p.map_scale;
  const int gmm = (1 << c.lgm) - 1;
  for (int side = 0; side < (c.two ? 1 : 2); ++side) {
    if (side == 1 && c.ring == 0) break;  // the equator is written once
    // Z[k] and Z[N - k] (natural order, chirped for Bluestein rings) of the
    // CTA's hemispheres, from W[k] and W[N - k]
    const int npairs = (N >> 1) + 1, nitems = npairs << c.lgm;
    // software pipeline over this thread's items: the first-term q of item
    // t + blockDim is in flight while item t is summed
    auto fetch = [&](int t, cplx (&qa)[2], cplx (&qb)[2]) {
      const int mi = t & gmm, kk = t >> c.lgm;
      const bool live = t < nitems && mi < c.nm;
      const double *qg = qbase + 2 * mi;
      first_term(qg, kk, mlim, qstride, half, live, qa[0], qb[0]);
      first_term(qg, N - kk, mlim, qstride, half, live && N - kk != kk, qa[1], qb[1]);
    };
    cplx qa[2], qb[2];
    fetch(threadIdx.x, qa, qb);
    for (int t = threadIdx.x; t < nitems; t += blockDim.x) {
      cplx na[2], nb[2];
      fetch(t + blockDim.x, na, nb);
      {
        const int mi = t & gmm, kk = t >> c.lgm, kr = N - kk;
        cplx Aa = {0.0, 0.0}, Ba = {0.0, 0.0}, Ab = {0.0, 0.0}, Bb = {0.0, 0.0};  // at kk and N - kk
        if (mi < c.nm) {
          const double *qg = qbase + 2 * mi;
          alias_sums(qg, kk, n, mlim, qstride, half, plo, phi, qa[0], qb[0], Aa, Ba);
          if (kr != kk) alias_sums(qg, kr, n, mlim, qstride, half, plo, phi, qa[1], qb[1], Ab, Bb);
          else { Ab = Aa; Bb = Ba; }
        }
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          if (h == 1 && !c.two) break;
          const int sd = c.two ? h : side;
          const double sgn = sd ? -1.0 : 1.0;
          const int g = (h << c.lgm) | mi;
          const cplx Wa = {Aa.x + sgn * Ba.x, Aa.y + sgn * Ba.y}, Wb = {Ab.x + sgn * Bb.x, Ab.y + sgn * Bb.y};
#pragma unroll
          for (int e = 0; e < 2; ++e) {
            const int k = e ? kr : kk;
            if (e && (kr == kk || kr == N)) break;
            cplx Wk = e ? Wb : Wa, Wc = cconj(e ? Wa : Wb);
            if (k == 0) {
              Wk.y = 0.0;
              Wc.y = 0.0;
            }
            const cplx sm = cadd(Wk, Wc), d = csub(Wk, Wc);
            const cplx Z = cadd(sm, mul_i(cmul(ring_root(p, c.R, k), d)));
            buf[at(k, g, lg)] = c.pow2 ? Z : cmul(Z, ring_chirp(p, c.R, k));
          }
        }
      }
      qa[0] = na[0];
      qa[1] = na[1];
      qb[0] = nb[0];
      qb[1] = nb[1];
    }
    if (!c.pow2)
      for (int t = threadIdx.x; t < ((M - N) << lg); t += blockDim.x)
        buf[at(N + (t >> lg), t & gm, lg)] = {0.0, 0.0};
    __syncthreads();
    auto sload = [&](int i, int g) -> cplx { return buf[at(i, g, lg)]; };
    auto sstore = [&](int i, int g, cplx v) { buf[at(i, g, lg)] = v; };
    auto out_row = [&](int g, int64_t pix) -> double * {
      const int64_t off = lane_side(c, g, side) ? c.R.off_south : c.R.off_north;
      return p.map + (off + pix) * p.nmaps + c.map0 + lane_map(c, g);
    };
    // pixels 2s, 2s + 1 of output z[s]; power of two: DIF position pos holds z[bitrev(pos)]
    auto pix_dif = [&](int pos, int g, cplx z) {
      if (!lane_live(c, g, side)) return;
      z = cscale(z, p.map_scale);
      const int64_t s2 = 2 * (int64_t)bitrev((unsigned)pos, c.bits);
      *out_row(g, s2) = z.x;
      *out_row(g, s2 + 1) = z.y;
    };
    auto pix_blue = [&](int k, int g, cplx z) {
      if (k >= N || !lane_live(c, g, side)) return;
      z = cscale(cmul(z, ring_chirp(p, c.R, k)), inv);
      *out_row(g, 2 * (int64_t)k) = z.x;
      *out_row(g, 2 * (int64_t)k + 1) = z.y;
    };
    if (c.pow2) {
      for (int ps = 0; ps < rs.n; ++ps) {
        if (ps == rs.n - 1) fft_pass_r<1, true>(fx, rs.r(ps), rs.lgl(ps), rs.wl(ps), sload, pix_dif);
        else fft_pass_r<1, true>(fx, rs.r(ps), rs.lgl(ps), rs.wl(ps), sload, sstore);
      }
    } else {
      for (int ps = 0; ps < rs.n - 1; ++ps)
        fft_pass_r<-1, true>(fx, rs.r(ps), rs.lgl(ps), rs.wl(ps), sload, sstore);
      const int R = rs.r(rs.n - 1);
      if (rs.n == 1) {
        bluestein_mid(fx, R, F, +1, 0, sload, pix_blue);
      } else {
        bluestein_mid(fx, R, F, +1, rs.wl(rs.n - 1), sload, sstore);
        for (int ps = rs.n - 2; ps >= 0; --ps) {
          if (rs.wl(ps) == 0 && rs.wl(ps + 1) != 0) __syncthreads();
          if (ps == 0) fft_pass_r<1, false>(fx, rs.r(ps), rs.lgl(ps), 0, sload, pix_blue);
          else fft_pass_r<1, false>(fx, rs.r(ps), rs.lgl(ps), rs.wl(ps), sload, sstore);
        }
      }
    }
    __syncthreads();  // the buffer is free for the other hemisphere
  }
}

__global__ void __launch_bounds__(kRingThreads, 1) k_ring_analysis(RingParams p) {
  extern __shared__ double smem_d[];
  const RingCta c = ring_cta(p, blockIdx.x);
  const int lg = c.lg, n = c.n, N = c.N, M = c.M;
  cplx *buf = reinterpret_cast<cplx *>(smem_d);
  cplx *plo = buf + ((int64_t)M << lg);
  cplx *phi = plo + kPhaseLo;
  phase_tables(plo, phi, p, c.ring);
  const int64_t half = p.nvecs, qstride = 2 * half;
  double *qbase = p.q_out + (int64_t)c.ring * (p.mmax + 1) * qstride + 2 * c.map0;
  const auto rs = radices<false>(M);
  const FftCtx fx{p.twiddles, ilog2(p.twlen), M, lg};
  const cplx *F = reinterpret_cast<const cplx *>(p.filters) + c.R.filter;
  const double inv = c.pow2 ? 1.0 : 1.0 / (double)M;
  const int gmm = (1 << c.lgm) - 1;
  const bool npow2 = (n & (n - 1)) == 0;  // every belt ring when nside is a power of two
  // 4 pi / npix, times the ring's quadrature weight when weights are set
  const double wscale = p.ring_weights ? p.scale * p.ring_weights[c.ring] : p.scale;
  // rows above the ring's m limit are written as zeros (null: every m folded)
  const int mlim = p.ring_mend ? p.ring_mend[c.ring] - 1 : p.mmax;
  for (int side = 0; side < (c.two ? 1 : 2); ++side) {
    if (side == 1 && c.ring == 0) break;
    auto in_row = [&](int g, int64_t pix) -> const double * {
      const int64_t off = lane_side(c, g, side) ? c.R.off_south : c.R.off_north;
      return p.map_in + (off + pix) * p.nmaps + c.map0 + lane_map(c, g);
    };
    auto sload = [&](int i, int g) -> cplx { return buf[at(i, g, lg)]; };
    auto sstore = [&](int i, int g, cplx v) { buf[at(i, g, lg)] = v; };
    // power of two: the DIT input position pos holds z[bitrev(pos)]
    auto pix_dit = [&](int pos, int g) -> cplx {
      if (!lane_live(c, g, side)) return {0.0, 0.0};
      const int64_t s2 = 2 * (int64_t)bitrev((unsigned)pos, c.bits);
      return {*in_row(g, s2), *in_row(g, s2 + 1)};
    };
    // Bluestein: chirped input z[k], zero beyond N
    auto pix_blue = [&](int k, int g) -> cplx {
      if (k >= N || !lane_live(c, g, side)) return {0.0, 0.0};
      const cplx z = {*in_row(g, 2 * (int64_t)k), *in_row(g, 2 * (int64_t)k + 1)};
      return cmul(z, cconj(ring_chirp(p, c.R, k)));
    };
    auto zstore = [&](int k, int g, cplx v) {
      if (k < N) buf[at(k, g, lg)] = cscale(cmul(v, cconj(ring_chirp(p, c.R, k))), inv);
    };
    if (c.pow2) {
      for (int ps = rs.n - 1; ps >= 0; --ps) {
        if (ps < rs.n - 1 && rs.wl(ps) == 0 && rs.wl(ps + 1) != 0) __syncthreads();
        if (ps == rs.n - 1) fft_pass_r<-1, false>(fx, rs.r(ps), rs.lgl(ps), rs.wl(ps), pix_dit, sstore);
        else fft_pass_r<-1, false>(fx, rs.r(ps), rs.lgl(ps), rs.wl(ps), sload, sstore);
      }
    } else {
      for (int ps = 0; ps < rs.n - 1; ++ps) {
        if (ps == 0) fft_pass_r<-1, true>(fx, rs.r(ps), rs.lgl(ps), 0, pix_blue, sstore);
        else fft_pass_r<-1, true>(fx, rs.r(ps), rs.lgl(ps), rs.wl(ps), sload, sstore);
      }
      const int R = rs.r(rs.n - 1);
      if (rs.n == 1) {
        bluestein_mid(fx, R, F, -1, 0, pix_blue, zstore);
      } else {
        bluestein_mid(fx, R, F, -1, rs.wl(rs.n - 1), sload, sstore);
        for (int ps = rs.n - 2; ps >= 0; --ps) {
          if (rs.wl(ps) == 0 && rs.wl(ps + 1) != 0) __syncthreads();
          if (ps == 0) fft_pass_r<1, false>(fx, rs.r(ps), rs.lgl(ps), 0, sload, zstore);
          else fft_pass_r<1, false>(fx, rs.r(ps), rs.lgl(ps), rs.wl(ps), sload, sstore);
        }
      }
    }
    // fold the spectrum F[k] (k <= N, from Z in natural order) of a lane into
    // g_m = F[m mod n] or its mirror, times e^{-i m phi0} and the scale
    auto fold = [&](int m, int g) -> cplx {
      const int jm = npow2 ? (m & (n - 1)) : m % n;
      const bool mirror = jm > N;
      const int k = mirror ? n - jm : jm;
      const int k1 = k == N ? 0 : k, k2 = k == 0 ? 0 : N - k;
      const cplx Zk = buf[at(k1, g, lg)];
      const cplx Zc = cconj(buf[at(k2, g, lg)]);
      const cplx E = cscale(cadd(Zk, Zc), 0.5);
      const cplx D = csub(Zk, Zc);
      const cplx O = {0.5 * D.y, -0.5 * D.x};  // D / (2i)
      cplx Fk = cadd(E, cmul(cconj(ring_root(p, c.R, k)), O));
      if (mirror) Fk = cconj(Fk);
      return cscale(cmul(Fk, cconj(phase_at(plo, phi, m))), wscale);
    };
    for (int t = threadIdx.x; t < ((p.mmax + 1) << c.lgm); t += blockDim.x) {
      const int mi = t & gmm, m = t >> c.lgm;
      if (mi >= c.nm) continue;
      double *qe = qbase + m * qstride + 2 * mi;
      double *qo = qe + half;
      if (m > mlim) {
        // the Legendre step weighs these q~ rows by values below 1e-30
        if (c.two || side == 0) {
          st2(qe, 0.0, 0.0);
          st2(qo, 0.0, 0.0);
        }
        continue;
      }
      if (c.two) {
        // both hemispheres: q~_even = g_N + g_S, q~_odd = g_N - g_S (g_S = 0 at the equator)
        const cplx gN = fold(m, mi), gS = fold(m, (1 << c.lgm) | mi);
        st2(qe, gN.x + gS.x, gN.y + gS.y);
        st2(qo, gN.x - gS.x, gN.y - gS.y);
      } else {
        const cplx gv = fold(m, mi);
        if (side == 0) {
          st2(qe, gv.x, gv.y);
          st2(qo, gv.x, gv.y);
        } else {
          const cplx e = ld2(qe), o = ld2(qo);
          st2(qe, e.x + gv.x, e.y + gv.y);
          st2(qo, o.x - gv.x, o.y - gv.y);
        }
      }
    }
    __syncthreads();
  }
}

// Plan creation: per ring pair the phase factors e^{i m phi0} for m < 64 and
// m = 64 a, a < nphase_hi (ones when phi0 = 0).
__global__ void k_ring_phases(RingParams p) {
  const DevRing R = p.rings[blockIdx.x];
  double2 *dst = p.phases_out + (int64_t)blockIdx.x * (kPhaseLo + p.nphase_hi);
  for (int k = threadIdx.x; k < kPhaseLo + p.nphase_hi; k += blockDim.x) {
    const long long m = k < kPhaseLo ? k : (long long)(k - kPhaseLo) * kPhaseLo;
    const cplx v = R.phi_num != 0 ? expi_pi(m * R.phi_num, R.phi_den) : cplx{1.0, 0.0};
    dst[k] = make_double2(v.x, v.y);
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
  auto sload = [&](int i, int g) -> cplx { return buf[at(i, g, 0)]; };
  auto sstore = [&](int i, int g, cplx v) { buf[at(i, g, 0)] = v; };
  const auto rs = radices<true>(M);
  const FftCtx fx{p.twiddles, ilog2(p.twlen), M, 0};
  for (int ps = 0; ps < rs.n; ++ps)
    fft_pass_r<-1, true>(fx, rs.r(ps), rs.lgl(ps), 0, sload, sstore);
  cplx *F = reinterpret_cast<cplx *>(p.filters_out) + R.filter;
  for (int k = threadIdx.x; k < M; k += blockDim.x) F[k] = buf[at(k, 0, 0)];
}

template <class K>
cudaError_t launch_rings(K kernel, const RingParams &prm, cudaStream_t st) {
  if (prm.ntasks <= 0) return cudaSuccess;
  cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, prm.smem);
  if (e != cudaSuccess) return e;
  kernel<<<prm.ntasks, kRingThreads, prm.smem, st>>>(prm);
  return cudaGetLastError();
}

}  // namespace

int32_t ring_cta_smem(int64_t buffer_cplx, int32_t nphase_hi) {
  return (int32_t)((buffer_cplx + kPhaseLo + nphase_hi + 8) * 2 * sizeof(double));
}

cudaError_t launch_ring_synthesis(const RingParams &prm, cudaStream_t st) {
  return launch_rings(k_ring_synthesis, prm, st);
}

cudaError_t launch_ring_analysis(const RingParams &prm, cudaStream_t st) {
  return launch_rings(k_ring_analysis, prm, st);
}

__global__ void k_residual(const double *__restrict__ a, const double *__restrict__ b, double *__restrict__ y,
                           int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    y[i] = a[i] - b[i];
}

__global__ void k_accumulate(const double *__restrict__ x, double *__restrict__ y, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    y[i] += x[i];
}

// One warp per (ring, m) row pair: 2 nvecs doubles between the ring-side q
// and the exchange buffer.
__global__ void k_shard_exchange(const int64_t *__restrict__ tab, int64_t nrings, int32_t mcount, int32_t nvecs,
                                 const double *__restrict__ src, double *__restrict__ dst, int gather) {
  const int lane = threadIdx.x & 31;
  const int64_t n = nrings * mcount;
  for (int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n;
       i += ((int64_t)gridDim.x * blockDim.x) >> 5) {
    const int64_t rl = i / mcount, m = i % mcount;
    const int64_t ring_off = i * 2 * nvecs, x_off = tab[2 * m] + rl * tab[2 * m + 1];
    const double *s = src + (gather ? x_off : ring_off);
    double *d = dst + (gather ? ring_off : x_off);
    for (int v = lane; v < 2 * nvecs; v += 32) d[v] = s[v];
  }
}

cudaError_t launch_shard_exchange(const int64_t *tab, int64_t nrings, int32_t mcount, int32_t nvecs,
                                  const double *src, double *dst, int gather, cudaStream_t st) {
  const int64_t n = nrings * mcount;
  if (n <= 0) return cudaSuccess;
  k_shard_exchange<<<(unsigned)std::min<int64_t>((n + 7) / 8, 8192), 256, 0, st>>>(tab, nrings, mcount, nvecs, src,
                                                                                     dst, gather);
  return cudaGetLastError();
}

cudaError_t launch_residual(const double *a, const double *b, double *y, int64_t n, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  k_residual<<<(unsigned)std::min<int64_t>((n + 255) / 256, 8192), 256, 0, st>>>(a, b, y, n);
  return cudaGetLastError();
}

cudaError_t launch_accumulate(const double *x, double *y, int64_t n, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  k_accumulate<<<(unsigned)std::min<int64_t>((n + 255) / 256, 8192), 256, 0, st>>>(x, y, n);
  return cudaGetLastError();
}

cudaError_t launch_ring_setup(const RingParams &prm, double *twiddles, double *filters, double *aux,
                              double2 *phases, cudaStream_t st) {
  k_twiddles<<<64, 256, 0, st>>>(reinterpret_cast<double2 *>(twiddles), prm.twlen);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  RingParams q = prm;
  q.phases_out = phases;
  k_ring_phases<<<prm.ni, 128, 0, st>>>(q);
  if ((e = cudaGetLastError()) != cudaSuccess || !filters) return e;
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
