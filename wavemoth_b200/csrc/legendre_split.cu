// Split-precision residual products of the butterfly Legendre step on the
// 5th-generation tensor cores (tcgen05.mma kind::i8, accumulators in TMEM).
//
// For one row group (see plan.h) the residual products are
//   alm2map   X[c][v] = sum_r P[r][c] a[r][v]     M = columns c, K = rows r
//   map2alm   a[r][v] = sum_c P[r][c] X[c][v]     M = rows r,    K = columns c
// with P generated in FP64 by the three-term recurrence of each column
// (src/legendre_transform.c.in:680-716), exactly as the FP64 kernels do.
//
// Ozaki-style splitting.  Each operand is scaled by a power of two so that
// its entries are at most 2^41 in magnitude along the GEMM's K dimension
// (P: per column for alm2map and per row for map2alm, fixed per plan; the
// alm / X operand: per group and vector, measured per call) and cut into six
// signed digits of 7 bits,
//   u = sum_i d_i 2^(35 - 7 i),   i = 0..5,   d_i in [-64, 64],
// with rounding error at most 1/2 (2^-42 relative to the scale).  The slice
// products with i + j <= 6 are accumulated exactly in int32 per diagonal
// D_k = sum_{i+j=k} A_i B_j (|D_k| <= 6 * 64^2 * K, far below 2^31 for the
// K of any HEALPix plan), and the epilogue forms
//   P a = 2^-(eA + eB) sum_k D_k 2^(70 - 7k)
// in FP64.  The dropped products (i + j >= 7) contribute at most 2^-46 of the
// scales.
//
// Tensor-core mapping.  D_k occupies TMEM columns [64k, 64k + 64) of a
// 512-column allocation (128 lanes = M).  The B operand slices of one chunk
// sit back to back in shared memory as one K-major operand of 384 rows, so
// one MMA of A_i against a window B_j0..B_j1 started at TMEM column
// 64 (i + j0) adds A_i B_j to D_{i+j} for every j of the window: nine MMAs
// per K step of 32 cover all 26 products, ordered so that the first MMA
// touching each TMEM column of a unit is an initialising one.
//
// Shared-memory operand layouts (no swizzle, 16-byte core-matrix rows):
//   K-major  (alm2map A, both B):  (mn / 8) SBO + (k / 16) 128 + (mn % 8) 16 + k % 16
//   MN-major (map2alm A):          (mn / 16) SBO + (k / 8) 128 + (k % 8) 16 + mn % 16
// A producer thread owns a 16-row segment of one column of P, started from
// the recurrence seeds stored every kSeedRows rows, and writes each slice of
// it as one 16-byte store in both layouts.  512 producer threads per CTA.
//
// Two ways to feed A:
//   * stored (default): the residual P of every tile is sliced once per plan
//     (k_res_slices_*) into device memory, and k_stream_split streams A and
//     B chunks with bulk copies; the level products (W sliced once per plan
//     by k_level_slices) always run this way;
//   * generated (WAVEMOTH_SPLIT_GENERATE, or too little device memory):
//     k_a2m_split / k_m2a_split produce P in the CTA.  Two stages: all
//     threads produce chunk t into stage t % 2 while the tensor core still
//     works on chunk t - 1; one thread issues the MMAs of a stage and commits
//     them to that stage's mbarrier, which the producers wait on before
//     refilling the stage.
// Both give the same slices and the same int32 accumulators.  Every wait is
// bounded: on expiry the kernel records kStatusTimeout, stops issuing work,
// waits (bounded) for its MMAs and copies, frees its TMEM and returns.
#include <cuda_runtime.h>

#include <algorithm>
#include <stdint.h>

#include "kernels.h"
#include "plan.h"

namespace wm {

namespace {

constexpr int kSplitThr = 512;
constexpr int kTmemCols = 512;
constexpr int kSplitDiag = 2 * kSplitSlices - 5;              // diagonals 0..6 kept
constexpr int kSliceA = kSplitM * kSplitK;                    // 8192 bytes
constexpr int kSliceB = kSplitN * kSplitK;                    // 4096
constexpr int kStageA = kSplitSlices * kSliceA;               // 49152
constexpr int kStageB = kSplitPlane;                          // 24576
constexpr int kXsStride = kSplitN + 1;  // epilogue tile row (doubles); odd: row-per-lane stores are free of bank conflicts
constexpr long long kWaitLimit = 1LL << 26;
static_assert(kSplitDiag * 64 <= kTmemCols, "diagonal accumulators exceed TMEM");
static_assert(kSplitM * kXsStride * 8 <= 2 * kStageA, "epilogue tile exceeds the A stages");

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// UMMA shared-memory descriptor, no swizzle (version 1 for sm_100).
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// Instruction descriptor of kind::i8: s32 accumulator, signed A and B,
// A K-major (a_mn = 0) or MN-major (a_mn = 1), B K-major, M = 128.
__device__ __forceinline__ uint32_t idesc_i8(int n, int a_mn) {
  return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)a_mn << 15) | ((uint32_t)(n >> 3) << 17) |
         ((uint32_t)(kSplitM >> 4) << 24);
}

__device__ __forceinline__ void mma_i8(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc,
                                       uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t phase) {
  uint32_t done = 0;
  for (long long it = 0; it < kWaitLimit; ++it) {
    asm volatile(
        "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(phase));
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void fence_operands() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void tmem_alloc(uint32_t *slot) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
               "r"((uint32_t)kTmemCols));
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
}
__device__ __forceinline__ void tmem_free(uint32_t base) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "r"((uint32_t)kTmemCols));
}

// 8 consecutive 32-bit TMEM columns of this thread's lane
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, int32_t (&v)[8]) {
  uint32_t r[8];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                 "=r"(r[7])
               : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int j = 0; j < 8; ++j) v[j] = (int32_t)r[j];
}

// Balanced base-128 digits of an integer |x| <= 2^20: x = a 2^14 + b 2^7 + c.
__device__ __forceinline__ void digits3(int x, int &a, int &b, int &c) {
  a = (x + 8192) >> 14;
  const int r = x - (a << 14);
  b = (r + 64) >> 7;
  c = r - (b << 7);
}

// Digits of u (|u| <= 2^41, an already scaled operand entry):
// u ~ sum_i d_i 2^(35 - 7 i), each digit in [-64, 64], error <= 1/2.  Two
// FP64 roundings to integers through the 1.5 * 2^52 shift (the integer is
// the low word of the sum), then integer digit extraction.
__device__ __forceinline__ void split_digits(double u, int (&d)[kSplitSlices]) {
  const double kShift = 6755399441055744.0;           // 1.5 * 2^52
  const double th = fma(u, 0x1p-21, kShift);
  const int hi = __double2loint(th);                   // rint(u / 2^21), |hi| <= 2^20
  const double rem = fma(-(th - kShift), 0x1p21, u);   // exact, |rem| <= 2^20
  const int lo = __double2loint(rem + kShift);         // rint(rem)
  digits3(hi, d[0], d[1], d[2]);
  digits3(lo, d[3], d[4], d[5]);
}

// Low bytes of four ints as one word (first argument in the lowest byte).
__device__ __forceinline__ uint32_t pack4(int a, int b, int c, int d) {
  const uint32_t ab = __byte_perm((uint32_t)a, (uint32_t)b, 0x0040);
  const uint32_t cd = __byte_perm((uint32_t)c, (uint32_t)d, 0x0040);
  return __byte_perm(ab, cd, 0x5410);
}

// Scale 2^e with max|x| 2^e <= 2^41 (1 for an all-zero operand).
__device__ __forceinline__ double2 operand_scale(double mx) {
  if (!(mx > 0.0)) return make_double2(1.0, 1.0);
  int e;
  frexp(mx, &e);  // mx < 2^e
  return make_double2(ldexp(1.0, 41 - e), ldexp(1.0, e - 41));
}

__device__ __forceinline__ int64_t alm_row0(const DevMatrix &M, int lmax) {
  return (int64_t)M.m * (2 * lmax - M.m + 3) / 2 + M.odd;
}

__device__ __forceinline__ double rec_step(const double *f64, const DevGCol &C, double x2, int r,
                                           double pc, double pp) {
  const double *ab = f64 + C.aux + 3 * (int64_t)(r - C.boff - 2);
  return (x2 + ab[0]) * ab[1] * pc + ab[2] * pp;
}

__device__ __forceinline__ void set_status(int32_t *status, int32_t code) {
  if (status) atomicCAS(status, 0, code);
}

}  // namespace
}  // namespace wm

namespace wm {
namespace {

// Group of a global column index (binary search over group column offsets).
__device__ __forceinline__ int group_of_col(const SplitParams &p, int64_t gc) {
  int lo = 0, hi = p.ngroups - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) / 2;
    if (p.groups[mid].cols <= gc) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// ------------------------------------------------------------------------
// Plan creation: max |P| per column (alm2map scale) and per row (map2alm
// scale), by running every column's recurrence over its rows.
// ------------------------------------------------------------------------
__global__ void k_split_maxima(SplitParams p) {
  const int64_t gc = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (gc >= p.ngcols) return;
  const int gi = group_of_col(p, gc);
  const DevGroup G = p.groups[gi];
  const DevSplitGroup S = p.sgroups[gi];
  const DevGCol C = p.gcols[gc];
  double mx = 0.0;
  if (C.start < G.nrows) {
    double pp = 0.0, pc = 0.0, x2 = 0.0;
    if (C.kind == 1) {
      x2 = p.f64[C.data];
      pp = p.f64[C.data + C.nx];
      pc = p.f64[C.data + 2 * C.nx];
    }
    for (int r = C.start; r < G.nrows; ++r) {
      double val;
      if (C.kind == 0) {
        val = p.f64[C.data + (r - C.start)];
      } else if (r == C.start) {
        val = pp;
      } else if (r == C.start + 1) {
        val = pc;
      } else {
        const double nv = rec_step(p.f64, C, x2, r, pc, pp);
        pp = pc;
        pc = nv;
        val = nv;
      }
      const double a = fabs(val);
      mx = fmax(mx, a);
      atomicMax(p.rowmax + S.rowoff + r, (unsigned long long)__double_as_longlong(a));
    }
  }
  p.colmax[gc] = (unsigned long long)__double_as_longlong(mx);
}

__global__ void k_split_scales(SplitParams p) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < p.ngcols) p.col_scale[i] = operand_scale(__longlong_as_double((long long)p.colmax[i]));
  if (i < p.nrowscale) p.row_scale[i] = operand_scale(__longlong_as_double((long long)p.rowmax[i]));
}

// ------------------------------------------------------------------------
// Operand pre-pass: per group (or root unit), the scale of every vector over
// the K range and the six slices of every K chunk, in the K-major layout of
// a B operand (kSplitN rows = vectors, kSplitK bytes of K per row).
//   kMode 0: K = group rows, entries a[arow0 + 2 (rs + r)][v0 + v]
//   kMode 1: K = group columns, entries X[row(c)][v0 + v]
//   kMode 2: K = s of a root (kT + kB), entries X[inT + s or inB + s - kT]
//   kMode 3: K = z of a root (n), entries q~[out_left + z]
// One CTA of 256 threads per group or root; thread (v, quarter) handles v.
// ------------------------------------------------------------------------
template <int kMode>
__device__ void slice_operand(const SplitParams &p, int gi) {
  __shared__ double red[4][kSplitN];
  __shared__ double2 sc[kSplitN];
  const int v = threadIdx.x & (kSplitN - 1), qtr = threadIdx.x >> 6;
  const int vn = min(kSplitN, p.nvecs - p.v0);
  DevGroup G{};
  DevPair P{};
  int K, nch;
  int64_t plane, sidx, rstride;
  const double *base;
  if (kMode <= 1) {
    G = p.groups[gi];
    const DevSplitGroup S = p.sgroups[gi];
    const DevMatrix M = p.mats[G.matrix];
    K = kMode == 0 ? G.nrows : G.ncols;
    nch = kMode == 0 ? S.nrchunks : S.ncchunks;
    plane = kMode == 0 ? S.apl : S.xpl;
    sidx = gi;
    if (kMode == 0) base = p.alm_in + alm_row0(M, p.lmax) * p.nvecs;
    else base = G.in_q ? p.q_in + (int64_t)(2 * M.m + M.odd) * p.q_mstride : p.xbuf + M.xrow * p.nvecs;
    rstride = (kMode == 1 && G.in_q) ? p.q_rstride : p.nvecs;
  } else {
    const DevRootUnit U = p.roots[gi];
    const DevSplitRoot R = p.sroots[gi];
    const DevMatrix M = p.mats[U.matrix];
    P = p.pairs[U.pair];
    K = kMode == 2 ? P.kT + P.kB : P.n;
    nch = kMode == 2 ? R.nsc : R.nzc;
    plane = kMode == 2 ? R.b_a2m : R.b_m2a;
    sidx = (int64_t)p.ngroups + gi;
    base = kMode == 2 ? p.xbuf + M.xrow * p.nvecs : p.q_in + (int64_t)(2 * M.m + M.odd) * p.q_mstride;
    rstride = kMode == 2 ? p.nvecs : p.q_rstride;
  }
  base += p.v0;
  auto entry = [&](int k) -> double {
    if (k >= K || v >= vn) return 0.0;
    int64_t row;
    if (kMode == 0) row = 2 * (int64_t)(G.rs + k);
    else if (kMode == 1) row = p.gcols[G.cols + k].row;
    else if (kMode == 2) row = k < P.kT ? P.inT + k : P.inB + (k - P.kT);
    else row = P.out_left + k;
    return base[row * rstride + v];
  };
  double mx = 0.0;
  // group columns (K up to the ring count, rows gathered through the column
  // table) keep sixteen rows' loads in flight per thread; the short ranges
  // of the other modes run faster with the compiler's own unrolling
  if constexpr (kMode == 1) {
#pragma unroll 16
    for (int k = qtr; k < K; k += 4) mx = fmax(mx, fabs(entry(k)));
  } else {
    for (int k = qtr; k < K; k += 4) mx = fmax(mx, fabs(entry(k)));
  }
  red[qtr][v] = mx;
  __syncthreads();
  if (qtr == 0) {
    const double m4 = fmax(fmax(red[0][v], red[1][v]), fmax(red[2][v], red[3][v]));
    sc[v] = operand_scale(m4);
    p.vec_scale[sidx * kSplitN + v] = sc[v];
  }
  __syncthreads();
  const double s = sc[v].x;
  int8_t *pl = p.planes + plane * (int64_t)kSplitPlane;
  auto slice_chunk = [&](int ch) {
    uint32_t w[kSplitSlices][4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      int d[4][kSplitSlices];
#pragma unroll
      for (int i = 0; i < 4; ++i) split_digits(entry(ch * kSplitK + qtr * 16 + 4 * j + i) * s, d[i]);
#pragma unroll
      for (int sl = 0; sl < kSplitSlices; ++sl) w[sl][j] = pack4(d[0][sl], d[1][sl], d[2][sl], d[3][sl]);
    }
    int8_t *dst = pl + (int64_t)ch * kSplitPlane + (v >> 3) * 512 + qtr * 128 + (v & 7) * 16;
#pragma unroll
    for (int sl = 0; sl < kSplitSlices; ++sl)
      *reinterpret_cast<uint4 *>(dst + sl * kSliceB) = make_uint4(w[sl][0], w[sl][1], w[sl][2], w[sl][3]);
  };
  if constexpr (kMode == 1) {
#pragma unroll 2
    for (int ch = 0; ch < nch; ++ch) slice_chunk(ch);
  } else {
    for (int ch = 0; ch < nch; ++ch) slice_chunk(ch);
  }
}

__global__ void __launch_bounds__(256) k_split_operand_alm(SplitParams p) {
  for (int gi = blockIdx.x; gi < p.ngroups; gi += gridDim.x) {
    slice_operand<0>(p, gi);
    __syncthreads();
  }
}

__global__ void __launch_bounds__(256) k_split_operand_x(SplitParams p) {
  for (int gi = blockIdx.x; gi < p.ngroups; gi += gridDim.x) {
    slice_operand<1>(p, gi);
    __syncthreads();
  }
}

// One warp per listed row: vectors [v0, v0 + kSplitN) of the row set to zero.
__global__ void __launch_bounds__(256) k_zero_rows(SplitParams p, const int64_t *rows, int32_t n) {
  const int vn = min(kSplitN, p.nvecs - p.v0);
  const int lane = threadIdx.x & 31;
  for (int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n;
       i += ((int64_t)gridDim.x * blockDim.x) >> 5) {
    const int64_t e = rows[i];
    const int buf = (int)(e >> kZeroBufShift);
    const int64_t row = e & ((1LL << kZeroBufShift) - 1);
    double *dst = (buf == 0 ? p.q : buf == 1 ? p.xbuf : p.alm_out) + row * p.nvecs + p.v0;
    for (int v = lane; v < vn; v += 32) dst[v] = 0.0;
  }
}

template <int kMode>
__global__ void __launch_bounds__(256) k_split_operand_level(SplitParams p) {
  for (int u = blockIdx.x; u < p.nroots; u += gridDim.x) {
    slice_operand<kMode>(p, u);
    __syncthreads();
  }
}

}  // namespace
}  // namespace wm

namespace wm {
namespace {

struct SplitSmem {
  uint64_t bar[2];
  uint32_t tmem;
  int32_t pad[3];
};

// The nine MMAs of one K step (32): A_i against windows of B_0..B_5 at TMEM
// column 64 (i + j0); the first three initialise columns [0, 256),
// [256, 384) and [384, 448) at the first step of a unit.
__device__ __forceinline__ void issue_step(uint32_t tmem, uint32_t a_base, uint32_t b_base, int a_mn,
                                           uint32_t a_lbo, uint32_t a_sbo, bool first) {
  const uint32_t init = first ? 0u : 1u;
  auto da = [&](int i) { return umma_desc(a_base + i * kSliceA, a_lbo, a_sbo); };
  auto db = [&](int j) { return umma_desc(b_base + j * kSliceB, 128, 512); };
  mma_i8(tmem + 0, da(0), db(0), idesc_i8(256, a_mn), init);      // D0..D3
  mma_i8(tmem + 256, da(0), db(4), idesc_i8(128, a_mn), init);    // D4, D5
  mma_i8(tmem + 384, da(2), db(4), idesc_i8(64, a_mn), init);     // D6
  mma_i8(tmem + 128, da(2), db(0), idesc_i8(256, a_mn), 1u);      // D2..D5
  mma_i8(tmem + 64, da(1), db(0), idesc_i8(256, a_mn), 1u);       // D1..D4
  mma_i8(tmem + 320, da(1), db(4), idesc_i8(128, a_mn), 1u);      // D5, D6
  mma_i8(tmem + 192, da(3), db(0), idesc_i8(256, a_mn), 1u);      // D3..D6
  mma_i8(tmem + 256, da(4), db(0), idesc_i8(192, a_mn), 1u);      // D4..D6
  mma_i8(tmem + 320, da(5), db(0), idesc_i8(128, a_mn), 1u);      // D5, D6
}

// FP64 value of the diagonal accumulators of one (lane, vector):
// 2^28 sum_k D_k 2^(42 - 7k), with the first and the second three diagonals
// combined exactly in 64-bit integers (|D_k| < 2^31), then two roundings.
__device__ __forceinline__ double recombine(const int32_t (&d)[kSplitDiag][8], int j) {
  const long long hi = ((long long)d[0][j] << 14) + ((long long)d[1][j] << 7) + d[2][j];
  const long long mid = ((long long)d[3][j] << 14) + ((long long)d[4][j] << 7) + d[5][j];
  return fma((double)hi, 0x1p28, fma((double)mid, 0x1p7, (double)d[6][j])) * 0x1p28;
}

// P at rows r0 .. r0 + 15 of group column c (zero outside [C.start, nrows)):
// dense values, or the recurrence from the seeds (P at s0 = max(r0, start)
// and s0 + 1) stored for the seed chunk of r0.  Returns false when the
// segment lies entirely outside the column's active rows (all zeros).
__device__ __forceinline__ bool column_segment(const SplitParams &p, const DevGroup &G, const DevGCol &C,
                                               int64_t c, int r0, double (&v)[16]) {
  if (C.start >= G.nrows || r0 >= G.nrows || r0 + 16 <= C.start) return false;
  if (C.kind == 1 && r0 >= C.start && r0 + 16 <= G.nrows) {
    // steady state: seeds at r0, r0 + 1, recurrence for the other 14 rows
    const double *seed = p.seeds + G.seeds + (c * G.nchunks + r0 / kSeedRows) * 2;
    double pp = seed[0], pc = seed[1];
    const double x2 = p.f64[C.data];
    const double *ab = p.f64 + C.aux + 3 * (int64_t)(r0 - C.boff);
    v[0] = pp;
    v[1] = pc;
#pragma unroll
    for (int i = 2; i < 16; ++i) {
      const double *a = ab + 3 * (i - 2);
      const double nv = (x2 + a[0]) * a[1] * pc + a[2] * pp;
      pp = pc;
      pc = nv;
      v[i] = nv;
    }
    return true;
  }
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = 0.0;
  if (C.kind == 0) {
#pragma unroll
    for (int i = 0; i < 16; ++i) {
      const int r = r0 + i;
      if (r >= C.start && r < G.nrows) v[i] = p.f64[C.data + (r - C.start)];
    }
    return true;
  }
  const int s0 = max(r0, C.start);
  const double *seed = p.seeds + G.seeds + (c * G.nchunks + r0 / kSeedRows) * 2;
  double pp = seed[0], pc = seed[1];
  const double x2 = p.f64[C.data];
  const double *ab = p.f64 + C.aux + 3 * (int64_t)(s0 - C.boff);  // coefficients of row s0 + 2
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    const int r = r0 + i;
    if (r < s0 || r >= G.nrows) continue;
    if (r == s0) {
      v[i] = pp;
    } else if (r == s0 + 1) {
      v[i] = pc;
    } else {
      const double *a = ab + 3 * (r - s0 - 2);
      const double nv = (x2 + a[0]) * a[1] * pc + a[2] * pp;
      pp = pc;
      pc = nv;
      v[i] = nv;
    }
  }
  return true;
}

// Scaled digits of 16 values, packed as four words per slice (row i in byte
// i % 4 of word i / 4), stored as one 16-byte row per slice.
__device__ __forceinline__ void store_zero_slices(unsigned char *dst) {
#pragma unroll
  for (int sl = 0; sl < kSplitSlices; ++sl) *reinterpret_cast<uint4 *>(dst + sl * kSliceA) = make_uint4(0, 0, 0, 0);
}

__device__ __forceinline__ void store_slices(unsigned char *dst, const double (&v)[16], const double *scale,
                                             int scale_stride) {
  uint32_t w[kSplitSlices][4];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    int d[4][kSplitSlices];
#pragma unroll
    for (int i = 0; i < 4; ++i) split_digits(v[4 * j + i] * scale[(4 * j + i) * scale_stride], d[i]);
#pragma unroll
    for (int sl = 0; sl < kSplitSlices; ++sl) w[sl][j] = pack4(d[0][sl], d[1][sl], d[2][sl], d[3][sl]);
  }
#pragma unroll
  for (int sl = 0; sl < kSplitSlices; ++sl)
    *reinterpret_cast<uint4 *>(dst + sl * kSliceA) = make_uint4(w[sl][0], w[sl][1], w[sl][2], w[sl][3]);
}

struct Pipe {
  uint32_t phase[2];
  bool pending[2];
  int stage;
};

// Waits (this thread) for the MMAs that last read the current stage; false on
// expiry.  The CTA agrees on the outcome at the next stage_issue.
__device__ __forceinline__ bool stage_free(SplitSmem *ss, Pipe &q) {
  const int s = q.stage;
  if (!q.pending[s]) return true;
  const bool ok = mbar_wait(&ss->bar[s], q.phase[s]);
  q.phase[s] ^= 1u;
  q.pending[s] = false;
  return ok;
}

// Waits for every outstanding MMA; false (CTA-uniform) on expiry.
__device__ __forceinline__ bool pipe_drain(SplitSmem *ss, Pipe &q) {
  bool ok = true;
  for (int s = 0; s < 2; ++s)
    if (q.pending[s]) {
      ok &= mbar_wait(&ss->bar[s], q.phase[s]);
      q.phase[s] ^= 1u;
      q.pending[s] = false;
    }
  return !__syncthreads_or(!ok);
}

// Starts the asynchronous copy of an operand-B chunk into the current stage.
__device__ __forceinline__ void stage_load_b(const SplitParams &p, unsigned char *smem, const Pipe &q, int64_t plane) {
  const unsigned char *src = reinterpret_cast<const unsigned char *>(p.planes) + plane * (int64_t)kSplitPlane;
  const uint32_t dst = smem_u32(smem + 2 * kStageA + q.stage * kStageB);
  for (int i = threadIdx.x; i < kStageB / 16; i += kSplitThr)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst + 16 * i), "l"(src + 16 * i) : "memory");
  asm volatile("cp.async.commit_group;" ::: "memory");
}

// Completes the stage (B copy, A stores of all threads), agrees on `ok`
// across the CTA, then (one thread) issues the two K steps of MMAs on it and
// commits them to the stage's mbarrier.  Returns false (CTA-uniform) if any
// thread's wait expired; no MMA is issued then.
__device__ __forceinline__ bool stage_issue(unsigned char *smem, SplitSmem *ss, Pipe &q, uint32_t tmem, int a_mn,
                                            bool first, bool ok) {
  asm volatile("cp.async.wait_group 0;" ::: "memory");
  fence_operands();
  if (__syncthreads_or(!ok)) return false;
  fence_after_sync();
  if (threadIdx.x == 0) {
    const uint32_t a0 = smem_u32(smem + q.stage * kStageA);
    const uint32_t b0 = smem_u32(smem + 2 * kStageA + q.stage * kStageB);
    for (int ks = 0; ks < kSplitK / 32; ++ks) {
      if (a_mn) issue_step(tmem, a0 + ks * 512, b0 + ks * 256, 1, 128, 1024, first && ks == 0);
      else issue_step(tmem, a0 + ks * 256, b0 + ks * 256, 0, 128, 512, first && ks == 0);
    }
    mma_commit(&ss->bar[q.stage]);
  }
  q.pending[q.stage] = true;
  q.stage ^= 1;
  return true;
}

// Epilogue: lane = M row of the unit; warps w, w + 4, w + 8, w + 12 share a
// TMEM lane quarter and take 16 vectors each.  Writes the FP64 tile into xs.
__device__ __forceinline__ void drain_tile(uint32_t tmem, double *xs, double row_inv, const double2 *vsc) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int row = 32 * (warp & 3) + lane;
  const uint32_t addr = tmem + ((uint32_t)(32 * (warp & 3)) << 16);
  for (int v8 = (warp >> 2) * 16; v8 < (warp >> 2) * 16 + 16; v8 += 8) {
    int32_t d[kSplitDiag][8];
#pragma unroll
    for (int k = 0; k < kSplitDiag; ++k) tmem_ld8(addr + 64 * k + v8, d[k]);
#pragma unroll
    for (int j = 0; j < 8; ++j) xs[row * kXsStride + v8 + j] = recombine(d, j) * row_inv * vsc[v8 + j].y;
  }
}

__device__ __forceinline__ SplitSmem *split_setup(unsigned char *smem) {
  SplitSmem *ss = reinterpret_cast<SplitSmem *>(smem + 2 * kStageA + 2 * kStageB);
  if ((threadIdx.x >> 5) == 0) tmem_alloc(&ss->tmem);
  if (threadIdx.x == 0) {
    mbar_init(&ss->bar[0], 1);
    mbar_init(&ss->bar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  return ss;
}

__device__ __forceinline__ void split_teardown(const SplitParams &p, SplitSmem *ss, Pipe &q, bool abort) {
  if (abort) {
    set_status(p.status, kStatusTimeout);
    for (int s = 0; s < 2; ++s)
      if (q.pending[s]) mbar_wait(&ss->bar[s], q.phase[s]);
  }
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  if ((threadIdx.x >> 5) == 0) tmem_free(ss->tmem);
}

// ------------------------------------------------------------------------
// alm2map residual.  Unit = <= 128 columns of one group; K chunks of 64 rows
// from the unit's first active chunk.  Thread t makes rows 16 (t >> 7) ..
// + 15 of each chunk for column col0 + (t & 127).
// ------------------------------------------------------------------------
__global__ void __launch_bounds__(kSplitThr, 1) k_a2m_split(SplitParams p) {
  extern __shared__ __align__(1024) unsigned char smem[];
  SplitSmem *ss = split_setup(smem);
  double2 *vsc = reinterpret_cast<double2 *>(ss + 1);
  double *xs = reinterpret_cast<double *>(smem);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int c = tid & (kSplitM - 1), seg = tid >> 7;
  const uint32_t tmem = ss->tmem;
  Pipe q{{0u, 0u}, {false, false}, 0};
  bool abort = false;
  for (int unit = blockIdx.x; unit < p.ntiles_a && !abort; unit += gridDim.x) {
    const DevSplitTileA T = p.tiles_a[unit];
    const DevGroup G = p.groups[T.group];
    const DevSplitGroup S = p.sgroups[T.group];
    const DevMatrix M = p.mats[G.matrix];
    if (tid < kSplitN) vsc[tid] = p.vec_scale[(int64_t)T.group * kSplitN + tid];
    const bool gen = c < T.ncols;
    const int64_t gc = (int64_t)T.col0 + c;
    DevGCol C{};
    double2 csc = make_double2(0.0, 0.0);
    if (gen) {
      C = p.gcols[G.cols + gc];
      csc = p.col_scale[G.cols + gc];
    } else {
      C.start = G.nrows;
    }
    for (int kc = T.kc0; kc < S.nrchunks; ++kc) {
      const bool ok = stage_free(ss, q);
      stage_load_b(p, smem, q, S.apl + kc);
      double v[16];
      unsigned char *dst = smem + q.stage * kStageA + (c >> 3) * 512 + seg * 128 + (c & 7) * 16;
      if (column_segment(p, G, C, gc, kc * kSplitK + 16 * seg, v)) store_slices(dst, v, &csc.x, 0);
      else store_zero_slices(dst);
      if (!stage_issue(smem, ss, q, tmem, 0, kc == T.kc0, ok)) {
        abort = true;
        break;
      }
    }
    if (abort || !pipe_drain(ss, q)) {
      abort = true;
      break;
    }
    fence_after_sync();
    drain_tile(tmem, xs,
               p.col_scale[G.cols + min((int64_t)T.col0 + 32 * (warp & 3) + lane, (int64_t)G.ncols - 1)].y,
               vsc);
    fence_before_sync();
    __syncthreads();
    {
      const int vn = min(kSplitN, p.nvecs - p.v0);
      double *base = G.in_q ? p.q + (int64_t)(2 * M.m + M.odd) * p.q_mstride : p.xbuf + M.xrow * p.nvecs;
      const int64_t rstride = G.in_q ? p.q_rstride : p.nvecs;
      for (int cc = warp; cc < T.ncols; cc += kSplitThr / 32) {
        const int row = p.gcols[G.cols + T.col0 + cc].row;
        const int vv = 2 * lane;
        if (vv < vn)
          *reinterpret_cast<double2 *>(base + (int64_t)row * rstride + p.v0 + vv) =
              make_double2(xs[cc * kXsStride + vv], xs[cc * kXsStride + vv + 1]);
      }
    }
    __syncthreads();
  }
  split_teardown(p, ss, q, abort);
}

// ------------------------------------------------------------------------
// map2alm residual.  Unit = <= 128 rows of one group, K = all its columns in
// chunks of 64.  Thread t makes rows 16 (t >> 6) .. + 15 of the unit for
// chunk column t & 63.
// ------------------------------------------------------------------------
__global__ void __launch_bounds__(kSplitThr, 1) k_m2a_split(SplitParams p) {
  extern __shared__ __align__(1024) unsigned char smem[];
  SplitSmem *ss = split_setup(smem);
  double2 *vsc = reinterpret_cast<double2 *>(ss + 1);
  double2 *rsc = vsc + kSplitN;
  double *xs = reinterpret_cast<double *>(smem);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int cl = tid & (kSplitK - 1), seg = tid >> 6;
  const uint32_t tmem = ss->tmem;
  Pipe q{{0u, 0u}, {false, false}, 0};
  bool abort = false;
  for (int unit = blockIdx.x; unit < p.ntiles_b && !abort; unit += gridDim.x) {
    const DevSplitTileB T = p.tiles_b[unit];
    const DevGroup G = p.groups[T.group];
    const DevSplitGroup S = p.sgroups[T.group];
    const DevMatrix M = p.mats[G.matrix];
    if (tid < kSplitN) vsc[tid] = p.vec_scale[(int64_t)T.group * kSplitN + tid];
    if (tid < kSplitM)
      rsc[tid] = tid < T.nrows ? p.row_scale[S.rowoff + T.row0 + tid] : make_double2(0.0, 0.0);
    __syncthreads();
    const int r0 = T.row0 + 16 * seg;
    for (int kc = 0; kc < S.ncchunks; ++kc) {
      const bool ok = stage_free(ss, q);
      stage_load_b(p, smem, q, S.xpl + kc);
      const int64_t gc = (int64_t)kc * kSplitK + cl;
      DevGCol C{};
      if (gc < G.ncols) C = p.gcols[G.cols + gc];
      else C.start = G.nrows;
      double v[16];
      unsigned char *dst = smem + q.stage * kStageA + seg * 1024 + (cl >> 3) * 128 + (cl & 7) * 16;
      if (column_segment(p, G, C, gc, r0, v)) store_slices(dst, v, &rsc[16 * seg].x, 2);
      else store_zero_slices(dst);
      if (!stage_issue(smem, ss, q, tmem, 1, kc == 0, ok)) {
        abort = true;
        break;
      }
    }
    if (abort || !pipe_drain(ss, q)) {
      abort = true;
      break;
    }
    fence_after_sync();
    drain_tile(tmem, xs, rsc[32 * (warp & 3) + lane].y, vsc);
    fence_before_sync();
    __syncthreads();
    {
      const int vn = min(kSplitN, p.nvecs - p.v0);
      const int64_t arow0 = alm_row0(M, p.lmax);
      for (int r = warp; r < T.nrows; r += kSplitThr / 32) {
        const int vv = 2 * lane;
        if (vv < vn)
          *reinterpret_cast<double2 *>(p.alm_out + (arow0 + 2 * (int64_t)(G.rs + T.row0 + r)) * p.nvecs +
                                       p.v0 + vv) =
              make_double2(xs[r * kXsStride + vv], xs[r * kXsStride + vv + 1]);
      }
    }
    __syncthreads();
  }
  split_teardown(p, ss, q, abort);
}

}  // namespace

namespace {

// W[z][s] of one interpolation block (k skeleton columns, n rows z): the unit
// vector of skeleton column s' at its row (filter 0), else column map[z] of
// the (n - k) x k interpolant (src/butterfly.c.in:222-235).
__device__ __forceinline__ double w_elem(const int32_t *map, const double *ip_t, int n, int k, int z, int s) {
  if (z >= n || s >= k) return 0.0;
  const int mt = map[z];
  if (mt < 0) return (s == -mt - 1) ? 1.0 : 0.0;
  return ip_t[mt + (int64_t)s * (n - k)];
}

// ------------------------------------------------------------------------
// Plan creation: W of every depth-1 root sliced into A chunks, for both
// directions (alm2map: rows z, K = s; map2alm: rows s, K = z), with a scale
// per row.  One CTA of 128 threads per level tile, thread = tile row.
// ------------------------------------------------------------------------
__global__ void __launch_bounds__(kSplitM) k_level_slices(SplitParams p) {
  const bool a2m = blockIdx.x < p.ntiles_la;
  const DevSplitLevelTile T = a2m ? p.tiles_la[blockIdx.x] : p.tiles_lm[blockIdx.x - p.ntiles_la];
  const DevRootUnit U = p.roots[T.unit];
  const DevPair P = p.pairs[U.pair];
  const DevSplitRoot R = p.sroots[T.unit];
  const int K = a2m ? P.kT + P.kB : P.n;
  const int nk = a2m ? R.nsc : R.nzc;
  const int r = threadIdx.x, row = T.row0 + r;
  const bool act = r < T.nrows;
  const int32_t *mapT = p.i32 + P.mapT, *mapB = p.i32 + P.mapB;
  const double *ipT = p.f64 + P.ipT_t, *ipB = p.f64 + P.ipB_t;
  auto w = [&](int k) -> double {
    if (!act || k >= K) return 0.0;
    const int z = a2m ? row : k, s = a2m ? k : row;
    return s < P.kT ? w_elem(mapT, ipT, P.n, P.kT, z, s) : w_elem(mapB, ipB, P.n, P.kB, z, s - P.kT);
  };
  double mx = 0.0;
  for (int k = 0; k < K; ++k) mx = fmax(mx, fabs(w(k)));
  const double2 sc = operand_scale(mx);
  if (act) p.level_rs[(a2m ? R.rs_a2m : R.rs_m2a) + row] = sc;
  int8_t *A = p.level_a + ((a2m ? R.a_a2m : R.a_m2a) + (int64_t)(T.row0 / kSplitM) * nk) * (int64_t)kStageA;
  for (int c = 0; c < nk; ++c) {
    for (int h = 0; h < kSplitK / 16; ++h) {
      double v[16];
#pragma unroll
      for (int i = 0; i < 16; ++i) v[i] = w(c * kSplitK + 16 * h + i);
      uint32_t wd[kSplitSlices][4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        int d[4][kSplitSlices];
#pragma unroll
        for (int i = 0; i < 4; ++i) split_digits(v[4 * j + i] * sc.x, d[i]);
#pragma unroll
        for (int sl = 0; sl < kSplitSlices; ++sl) wd[sl][j] = pack4(d[0][sl], d[1][sl], d[2][sl], d[3][sl]);
      }
      int8_t *dst = A + (int64_t)c * kStageA + (r >> 3) * 512 + h * 128 + (r & 7) * 16;
#pragma unroll
      for (int sl = 0; sl < kSplitSlices; ++sl)
        *reinterpret_cast<uint4 *>(dst + sl * kSliceA) = make_uint4(wd[sl][0], wd[sl][1], wd[sl][2], wd[sl][3]);
    }
  }
}

// One-dimensional bulk copy (TMA) into this CTA's own shared memory,
// completing on `bar`, and the arrival that announces its bytes.
__device__ __forceinline__ void bulk_load(uint32_t dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

// ------------------------------------------------------------------------
// Streamed split GEMM.  Both operands arrive pre-sliced from global memory
// (A chunks cut once per plan, B planes by the operand pre-pass), so one
// kernel serves the residual and level products of both directions.
// Warp roles (one CTA per SM, persistent over the tile list):
//   warp 0   one thread loads chunk after chunk with 1D bulk copies (TMA,
//            each into this CTA only) into kStreamStages stages, running ahead into the
//            next tile while the current one drains;
//   warp 1   one thread issues the nine MMAs per K step of 32 and commits
//            each stage back to the loader, the finished tile to the
//            epilogue;
//   warps 2..9 drain TMEM (warp w reads lane quarter w % 4, vector half
//            (w - 2) / 4), release it to the MMA thread, scale the FP64 tile
//            into shared memory and write its rows to global memory while
//            the next tile's MMAs run.
// Every wait is bounded and also gives up when another role has recorded an
// abort; the MMA thread then waits (bounded) for its MMAs and the loader for
// its copies before the CTA frees TMEM and returns.
// ------------------------------------------------------------------------
constexpr int kStreamStages = 2;
constexpr int kStreamEpiWarps = 8;
constexpr int kStreamThr = 32 * (2 + kStreamEpiWarps);
constexpr int kStreamStage = kStageA + kStageB;  // 73728 bytes

struct StreamSmem {
  uint64_t full[kStreamStages], empty[kStreamStages];
  uint64_t acc_full, acc_empty, fin;
  uint32_t tmem;
  int32_t abort;
};

// Bounded wait (at most `limit` polls) that also ends when *abort is set;
// false unless completed.  The waits for progress of another role use the
// plan's limit; the drains before exit keep kWaitLimit (copies and MMAs
// already issued always complete in hardware).
__device__ __forceinline__ bool mbar_wait_or_abort(uint64_t *bar, uint32_t phase, volatile int32_t *abort,
                                                   long long limit) {
  uint32_t done = 0;
  for (long long it = 0; it < limit; ++it) {
    asm volatile(
        "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(phase));
    if (done) return true;
    if ((it & 255) == 255 && *abort) return false;
  }
  *abort = 1;
  return false;
}

// Barrier 1 over the epilogue warps with an OR of `v` (the same answer in
// every epilogue thread, so they leave their loop together).
__device__ __forceinline__ bool epi_sync_or(bool v) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\tsetp.ne.u32 p, %1, 0;\n\t"
      "bar.red.or.pred q, 1, %2, p;\n\tselp.u32 %0, 1, 0, q;\n\t}\n"
      : "=r"(r)
      : "r"((uint32_t)v), "n"(32 * kStreamEpiWarps)
      : "memory");
  return r != 0;
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// 7 x 8 TMEM columns (the diagonals of 8 vectors) of this thread's lane with
// one wait.
__device__ __forceinline__ void tmem_ld_diags(uint32_t taddr, int32_t (&d)[kSplitDiag][8]) {
#pragma unroll
  for (int k = 0; k < kSplitDiag; ++k) {
    uint32_t r[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                   "=r"(r[7])
                 : "r"(taddr + 64 * k));
#pragma unroll
    for (int j = 0; j < 8; ++j) d[k][j] = (int32_t)r[j];
  }
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

template <int kAmn>
__global__ void __launch_bounds__(kStreamThr, 1) k_stream_split(SplitParams p, StreamLaunch L) {
  extern __shared__ __align__(1024) unsigned char smem[];
  StreamSmem *ss = reinterpret_cast<StreamSmem *>(smem + kStreamStages * kStreamStage);
  double *xs = reinterpret_cast<double *>(smem + kStreamStages * kStreamStage + 128);
  double *erinv = xs + kSplitM * kXsStride;  // epilogue: 1 / scale of each tile row,
  double *evs = erinv + kSplitM;             // 1 / scale of each vector,
  int32_t *erow = reinterpret_cast<int32_t *>(evs + kSplitN);  // destination row of each tile row
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  volatile int32_t *abort = &ss->abort;
  const long long lim = p.wait_limit > 0 ? p.wait_limit : kWaitLimit;
  if (warp == 0) tmem_alloc(&ss->tmem);
  if (tid == 0) {
    for (int s = 0; s < kStreamStages; ++s) {
      mbar_init(&ss->full[s], 1);
      mbar_init(&ss->empty[s], 1);
    }
    mbar_init(&ss->acc_full, 1);
    mbar_init(&ss->acc_empty, kStreamEpiWarps);
    mbar_init(&ss->fin, 1);
    ss->abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = ss->tmem;
  if (warp == 0) {
    // ---------------- loader ----------------
    if (lane == 0) {
      long long g = 0;  // chunks issued
      DevStreamTile Tn{};
      if (blockIdx.x < L.ntiles) Tn = L.tiles[blockIdx.x];
      for (int t = blockIdx.x; t < L.ntiles && !*abort; t += gridDim.x) {
        const DevStreamTile T = Tn;
        if (t + (int)gridDim.x < L.ntiles) Tn = L.tiles[t + gridDim.x];  // next descriptor in flight
        for (int c = 0; c < T.nk; ++c, ++g) {
          const int s = (int)(g % kStreamStages);
          const long long use = g / kStreamStages;
          if (use > 0 && !mbar_wait_or_abort(&ss->empty[s], (uint32_t)((use - 1) & 1), abort, lim)) break;
          const uint32_t dst = smem_u32(smem + s * kStreamStage);
          expect_tx(&ss->full[s], kStreamStage);
          bulk_load(dst, L.a + (T.a + c) * (int64_t)kStageA, kStageA, &ss->full[s]);
          bulk_load(dst + kStageA, p.planes + (T.b + c) * (int64_t)kSplitPlane, kStageB, &ss->full[s]);
        }
      }
      // every issued copy lands before the CTA may exit
      for (int s = 0; s < kStreamStages; ++s) {
        const long long n = g > s ? (g - 1 - s) / kStreamStages + 1 : 0;  // copies into stage s
        if (n > 0) mbar_wait(&ss->full[s], (uint32_t)((n - 1) & 1));
      }
    }
    __syncwarp();
  } else if (warp == 1) {
    // ---------------- MMA issue ----------------
    if (lane == 0) {
      long long g = 0;
      int nt = 0;
      for (int t = blockIdx.x; t < L.ntiles && !*abort; t += gridDim.x, ++nt) {
        const DevStreamTile T = L.tiles[t];
        if (nt > 0 && !mbar_wait_or_abort(&ss->acc_empty, (uint32_t)((nt - 1) & 1), abort, lim)) break;
        fence_after_sync();
        bool ok = true;
        for (int c = 0; c < T.nk; ++c, ++g) {
          const int s = (int)(g % kStreamStages);
          if (!mbar_wait_or_abort(&ss->full[s], (uint32_t)((g / kStreamStages) & 1), abort, lim)) {
            ok = false;
            break;
          }
          fence_after_sync();
          const uint32_t a0 = smem_u32(smem + s * kStreamStage), b0 = a0 + kStageA;
          for (int ks = 0; ks < kSplitK / 32; ++ks) {
            if (kAmn) issue_step(tmem, a0 + ks * 512, b0 + ks * 256, 1, 128, 1024, c == 0 && ks == 0);
            else issue_step(tmem, a0 + ks * 256, b0 + ks * 256, 0, 128, 512, c == 0 && ks == 0);
          }
          mma_commit(&ss->empty[s]);
        }
        if (!ok) break;
        mma_commit(&ss->acc_full);
      }
      // every issued MMA completes before TMEM and shared memory are released
      mma_commit(&ss->fin);
      mbar_wait(&ss->fin, 0);
    }
    __syncwarp();
  } else {
    // ---------------- epilogue ----------------
    const int qd = warp & 3, half = (warp - 2) >> 2;
    const int row = 32 * qd + lane;
    const uint32_t addr = tmem + ((uint32_t)(32 * qd) << 16);
    const int etid = tid - 64;
    const int vn = min(kSplitN, p.nvecs - p.v0);
    int nt = 0;
    for (int t = blockIdx.x; t < L.ntiles; t += gridDim.x, ++nt) {
      const DevStreamTile T = L.tiles[t];
      // the tile's row map and scales, fetched while its MMAs still run (the
      // previous tile's rows were all written before the last barrier)
      if (etid < kSplitM) {
        const int64_t e = (int64_t)t * kSplitM + etid;
        erow[etid] = L.rows[e];
        const int32_t si = L.sidx[e];
        erinv[etid] = si >= 0 ? L.scales[si].y : 0.0;
      } else if (etid < kSplitM + kSplitN) {
        evs[etid - kSplitM] = p.vec_scale[(int64_t)T.vs * kSplitN + etid - kSplitM].y;
      }
      const bool ok = mbar_wait_or_abort(&ss->acc_full, (uint32_t)(nt & 1), abort, lim);
      if (epi_sync_or(!ok || *abort)) break;
      fence_after_sync();
      const double rinv = erinv[row];
      for (int v8 = 32 * half; v8 < 32 * half + 32; v8 += 8) {
        int32_t d[kSplitDiag][8];
        tmem_ld_diags(addr + v8, d);
#pragma unroll
        for (int j = 0; j < 8; ++j) xs[row * kXsStride + v8 + j] = recombine(d, j) * rinv * evs[v8 + j];
      }
      // TMEM is free for the next tile once every epilogue warp has read it
      fence_before_sync();
      __syncwarp();
      if (lane == 0) mbar_arrive(&ss->acc_empty);
      asm volatile("bar.sync 1, %0;" ::"n"(32 * kStreamEpiWarps));
      double *dbase = T.buf == 0 ? p.q : T.buf == 1 ? p.xbuf : p.alm_out;
      for (int r = etid >> 5; r < kSplitM; r += kStreamEpiWarps) {
        const int32_t dr = erow[r];
        const int vv = 2 * lane;
        if (dr >= 0 && vv < vn)
          *reinterpret_cast<double2 *>(dbase + (int64_t)dr * p.nvecs + p.v0 + vv) =
              make_double2(xs[r * kXsStride + vv], xs[r * kXsStride + vv + 1]);
      }
      asm volatile("bar.sync 1, %0;" ::"n"(32 * kStreamEpiWarps));
    }
  }
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  if (*abort) set_status(p.status, kStatusTimeout);
  if (warp == 0) tmem_free(tmem);
}

// ------------------------------------------------------------------------
// Plan creation: residual P of the split tiles sliced once into A chunks in
// the layouts the on-the-fly kernels build in shared memory (alm2map
// K-major, map2alm MN-major), from the same recurrence seeds and scales, so
// the streamed GEMM sees exactly the slices those kernels would generate.
// One CTA of 512 threads per tile, all its K chunks.
// ------------------------------------------------------------------------
__global__ void __launch_bounds__(kSplitThr) k_res_slices_a2m(SplitParams p, StreamLaunch L) {
  const int t = blockIdx.x;
  const DevSplitTileA T = p.tiles_a[t];
  const DevStreamTile ST = L.tiles[t];
  const DevGroup G = p.groups[T.group];
  const DevSplitGroup S = p.sgroups[T.group];
  const int tid = threadIdx.x, c = tid & (kSplitM - 1), seg = tid >> 7;
  const int64_t gc = (int64_t)T.col0 + c;
  DevGCol C{};
  double2 csc = make_double2(0.0, 0.0);
  if (c < T.ncols) {
    C = p.gcols[G.cols + gc];
    csc = p.col_scale[G.cols + gc];
  } else {
    C.start = G.nrows;
  }
  unsigned char *A = reinterpret_cast<unsigned char *>(const_cast<int8_t *>(L.a)) + ST.a * (int64_t)kStageA;
  for (int kc = T.kc0; kc < S.nrchunks; ++kc) {
    unsigned char *dst = A + (int64_t)(kc - T.kc0) * kStageA + (c >> 3) * 512 + seg * 128 + (c & 7) * 16;
    double v[16];
    if (column_segment(p, G, C, gc, kc * kSplitK + 16 * seg, v)) store_slices(dst, v, &csc.x, 0);
    else store_zero_slices(dst);
  }
}

__global__ void __launch_bounds__(kSplitThr) k_res_slices_m2a(SplitParams p, StreamLaunch L) {
  __shared__ double2 rsc[kSplitM];
  const int t = blockIdx.x;
  const DevSplitTileB T = p.tiles_b[t];
  const DevStreamTile ST = L.tiles[t];
  const DevGroup G = p.groups[T.group];
  const DevSplitGroup S = p.sgroups[T.group];
  const int tid = threadIdx.x, cl = tid & (kSplitK - 1), seg = tid >> 6;
  if (tid < kSplitM) rsc[tid] = tid < T.nrows ? p.row_scale[S.rowoff + T.row0 + tid] : make_double2(0.0, 0.0);
  __syncthreads();
  const int r0 = T.row0 + 16 * seg;
  unsigned char *A = reinterpret_cast<unsigned char *>(const_cast<int8_t *>(L.a)) + ST.a * (int64_t)kStageA;
  for (int kc = 0; kc < S.ncchunks; ++kc) {
    const int64_t gc = (int64_t)kc * kSplitK + cl;
    DevGCol C{};
    if (gc < G.ncols) C = p.gcols[G.cols + gc];
    else C.start = G.nrows;
    unsigned char *dst = A + (int64_t)kc * kStageA + seg * 1024 + (cl >> 3) * 128 + (cl & 7) * 16;
    double v[16];
    if (column_segment(p, G, C, gc, r0, v)) store_slices(dst, v, &rsc[16 * seg].x, 2);
    else store_zero_slices(dst);
  }
}

}  // namespace

static size_t stream_smem_bytes() {
  return (size_t)kStreamStages * kStreamStage + 128 + (size_t)kSplitM * kXsStride * 8 +
         (kSplitM + kSplitN) * sizeof(double) + kSplitM * sizeof(int32_t);
}

cudaError_t launch_stream(const SplitParams &prm, const StreamLaunch &L, int grid, cudaStream_t st) {
  if (L.ntiles <= 0) return cudaSuccess;
  const size_t sm = stream_smem_bytes();
  cudaError_t e;
  if (L.a_mn) {
    e = cudaFuncSetAttribute(k_stream_split<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    k_stream_split<1><<<grid, kStreamThr, sm, st>>>(prm, L);
  } else {
    e = cudaFuncSetAttribute(k_stream_split<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    k_stream_split<0><<<grid, kStreamThr, sm, st>>>(prm, L);
  }
  return cudaGetLastError();
}

cudaError_t launch_residual_slices(const SplitParams &prm, const StreamLaunch &a2m, const StreamLaunch &m2a,
                                   cudaStream_t st) {
  if (a2m.ntiles > 0) k_res_slices_a2m<<<a2m.ntiles, kSplitThr, 0, st>>>(prm, a2m);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  if (m2a.ntiles > 0) k_res_slices_m2a<<<m2a.ntiles, kSplitThr, 0, st>>>(prm, m2a);
  return cudaGetLastError();
}

cudaError_t launch_level_slices(const SplitParams &prm, cudaStream_t st) {
  const int n = prm.ntiles_la + prm.ntiles_lm;
  if (n == 0) return cudaSuccess;
  k_level_slices<<<n, kSplitM, 0, st>>>(prm);
  return cudaGetLastError();
}

// dynamic shared memory of the split GEMM kernels
static size_t split_smem_bytes() {
  return (size_t)2 * kStageA + 2 * kStageB + sizeof(SplitSmem) + (kSplitN + kSplitM) * sizeof(double2);
}

cudaError_t launch_split(int which, const SplitParams &prm, int grid, cudaStream_t st) {
  cudaError_t e = cudaSuccess;
  switch (which) {
    case 0:
      k_split_operand_alm<<<grid, 256, 0, st>>>(prm);
      break;
    case 2:
      k_split_operand_x<<<grid, 256, 0, st>>>(prm);
      break;
    case 1:
    case 3: {
      const size_t sm = split_smem_bytes();
      if (which == 1) {
        e = cudaFuncSetAttribute(k_a2m_split, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e != cudaSuccess) return e;
        k_a2m_split<<<grid, kSplitThr, sm, st>>>(prm);
      } else {
        e = cudaFuncSetAttribute(k_m2a_split, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e != cudaSuccess) return e;
        k_m2a_split<<<grid, kSplitThr, sm, st>>>(prm);
      }
      break;
    }
    case 4:
      k_split_operand_level<2><<<grid, 256, 0, st>>>(prm);
      break;
    case 6:
      k_split_operand_level<3><<<grid, 256, 0, st>>>(prm);
      break;
    default:
      return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_zero_rows(const SplitParams &prm, const int64_t *rows, int32_t n, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  const int grid = (int)std::min<int64_t>(((int64_t)n + 7) / 8, 4096);
  k_zero_rows<<<grid, 256, 0, st>>>(prm, rows, n);
  return cudaGetLastError();
}

cudaError_t launch_split_scales(const SplitParams &prm, cudaStream_t st) {
  if (prm.ngcols == 0) return cudaSuccess;
  const int block = 128;
  k_split_maxima<<<(unsigned)((prm.ngcols + block - 1) / block), block, 0, st>>>(prm);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  const int64_t n = prm.ngcols > prm.nrowscale ? prm.ngcols : prm.nrowscale;
  k_split_scales<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(prm);
  return cudaGetLastError();
}

}  // namespace wm
