// FP64 butterfly Legendre kernels (the plain path).
//
// alm2map, per (m, parity) matrix:  q = A^T a  with  A = D S_L ... S_1
//   1. residual stage   depth-0 buffer rows  = D^T a, one row per skeleton
//                       column of every root block: a three-term recurrence
//                       down the rows of each column (or a dense column)
//                       (src/wavemoth.c:958-1009, legendre_transform.c.in:680-716)
//   2. level t = 0..L-1 lower rows = S^T applied to the upper rows: each
//                       lower row is the sum of a T and a B term, each either
//                       a copy of a skeleton row or a dot product of an
//                       interpolant column with the skeleton rows
//                       (src/butterfly.c.in:222-235, :284-373)
//   The lower buffer of the last level is q itself (rows = rings).
//
// map2alm, per matrix:  a = A q~  (the exact adjoint, applied leaves -> root:
//   butterfly.pyx:258-264 for one interpolation block, then the transpose of
//   the residual stage, done as "recurrence tile in shared memory, then a
//   small matrix product" so that every column's recurrence runs once).
//
// Work distribution: a persistent grid; each CTA pulls matrix indices from a
// global counter (largest matrices first, order chosen on the host) and
// processes one matrix at a time with all its threads; level buffers live in
// a per-CTA slot of global scratch (L2 resident).  Every output element has
// exactly one writer and a fixed summation order, so results are bitwise
// reproducible run to run.
#include <cuda_runtime.h>
#include <stdint.h>

#include "plan.h"
#include "kernels.h"

namespace wm {

namespace {

constexpr int kThreads = 256;
constexpr int kRowChunk = 16;   // map2alm residual: rows per recurrence tile

template <int VC>
__device__ __forceinline__ void load_vec(double (&x)[VC], const double *p, int nv) {
#pragma unroll
  for (int v = 0; v < VC; ++v) x[v] = (v < nv) ? p[v] : 0.0;
}

__device__ __forceinline__ int next_matrix(int32_t *counter, int *s_idx) {
  __syncthreads();
  if (threadIdx.x == 0) *s_idx = atomicAdd(counter, 1);
  __syncthreads();
  return *s_idx;
}

__device__ __forceinline__ int64_t alm_row0(const DevMatrix &M, int lmax) {
  // alm row of matrix row 0 (l = m + odd) in the m-major layout
  return (int64_t)M.m * (2 * lmax - M.m + 3) / 2 + M.odd;
}

template <int VC>
__global__ void __launch_bounds__(kThreads) k_alm2map_legendre(LegendreParams p) {
  __shared__ int s_idx;
  double *A = p.scratch + (int64_t)blockIdx.x * p.slot_stride;
  double *B = A + p.slot_stride / 2;
  const int nvecs = p.nvecs;
  const int nvc = (nvecs + VC - 1) / VC;
  const int64_t astep = 2 * (int64_t)nvecs;  // every other alm row
  for (;;) {
    int idx = next_matrix(p.counter, &s_idx);
    if (idx >= p.nmats) break;
    const DevMatrix M = p.mats[p.order[idx]];
    double *qm = p.q_out + (int64_t)(2 * M.m + M.odd) * p.q_mstride;
    double *level0 = M.nlevels > 0 ? A : qm;
    const int64_t l0s = M.nlevels > 0 ? nvecs : p.q_rstride;  // row stride of level0
    const int64_t arow0 = alm_row0(M, p.lmax);

    // ---- residual stage: one item per (depth-0 row, vector chunk) ----
    const int32_t *rmap = p.i32 + M.root_map;
    const int nitems = p.level0_given ? 0 : M.root_rows * nvc;
    for (int it = threadIdx.x; it < nitems; it += blockDim.x) {
      const int row = it % M.root_rows, v0 = (it / M.root_rows) * VC;
      const int nv = min(VC, nvecs - v0);
      const DevStrip S = p.strips[rmap[2 * row]];
      const int c = rmap[2 * row + 1];
      const DevDBlock D = p.dblocks[S.dblock];
      const int nks = D.nrows - S.rstart;
      const double *a = p.alm_in + (arow0 + 2 * (int64_t)(D.row_start + S.rstart)) * nvecs + v0;
      double acc[VC];
#pragma unroll
      for (int v = 0; v < VC; ++v) acc[v] = 0.0;
      if (S.kind == 0) {
        const double *col = p.f64 + S.data + (int64_t)c * nks;
        for (int kk = 0; kk < nks; ++kk) {
          double x[VC];
          load_vec<VC>(x, a + kk * astep, nv);
          const double pv = col[kk];
#pragma unroll
          for (int v = 0; v < VC; ++v) acc[v] += pv * x[v];
        }
      } else {
        const int nx = S.cstop - S.cstart;
        const double *base = p.f64 + S.data;
        const double x2 = base[c];
        double pp = base[nx + c], pc = base[2 * nx + c];
        double x[VC];
        load_vec<VC>(x, a, nv);
#pragma unroll
        for (int v = 0; v < VC; ++v) acc[v] += pp * x[v];
        load_vec<VC>(x, a + astep, nv);
#pragma unroll
        for (int v = 0; v < VC; ++v) acc[v] += pc * x[v];
        const double *aux = p.f64 + D.aux + 3 * (int64_t)S.rstart;
        for (int kl = 2; kl < nks; ++kl) {
          const double *ab = aux + 3 * (kl - 2);
          const double nv2 = (x2 + ab[0]) * ab[1] * pc + ab[2] * pp;
          pp = pc;
          pc = nv2;
          load_vec<VC>(x, a + kl * astep, nv);
#pragma unroll
          for (int v = 0; v < VC; ++v) acc[v] += nv2 * x[v];
        }
      }
      double *out = level0 + (int64_t)row * l0s + v0;
#pragma unroll
      for (int v = 0; v < VC; ++v)
        if (v < nv) out[v] = acc[v];
    }
    __syncthreads();

    // ---- interpolation levels, root side to leaf side ----
    for (int t = 0; t < M.nlevels; ++t) {
      const DevLevel L = p.levels[M.level_begin + t];
      const double *upper = (t & 1) ? B : A;
      double *lower = (t == M.nlevels - 1) ? qm : ((t & 1) ? A : B);
      const int64_t lws = (t == M.nlevels - 1) ? p.q_rstride : nvecs;  // row stride of lower
      const int32_t *lm = p.i32 + L.lower_map;
      const int n_items = L.lower_rows * nvc;
      for (int it = threadIdx.x; it < n_items; it += blockDim.x) {
        const int row = it % L.lower_rows, v0 = (it / L.lower_rows) * VC;
        const int nv = min(VC, nvecs - v0);
        const DevPair P = p.pairs[lm[2 * row]];
        const int z = lm[2 * row + 1];
        double acc[VC];
#pragma unroll
        for (int v = 0; v < VC; ++v) acc[v] = 0.0;
#pragma unroll
        for (int side = 0; side < 2; ++side) {
          const int k = side ? P.kB : P.kT;
          const int in = side ? P.inB : P.inT;
          const int mt = p.i32[(side ? P.mapB : P.mapT) + z];
          const double *src = upper + (int64_t)in * nvecs + v0;
          double x[VC];
          if (mt < 0) {
            load_vec<VC>(x, src + (int64_t)(-mt - 1) * nvecs, nv);
#pragma unroll
            for (int v = 0; v < VC; ++v) acc[v] += x[v];
          } else {
            const int nmk = P.n - k;
            const double *w = p.f64 + (side ? P.ipB_t : P.ipT_t) + mt;
            for (int s = 0; s < k; ++s) {
              const double ws = w[(int64_t)s * nmk];
              load_vec<VC>(x, src + (int64_t)s * nvecs, nv);
#pragma unroll
              for (int v = 0; v < VC; ++v) acc[v] += ws * x[v];
            }
          }
        }
        double *out = lower + (int64_t)row * lws + v0;
#pragma unroll
        for (int v = 0; v < VC; ++v)
          if (v < nv) out[v] = acc[v];
      }
      __syncthreads();
    }
  }
}

template <int VC>
__global__ void __launch_bounds__(kThreads) k_map2alm_legendre(LegendreParams p) {
  __shared__ int s_idx;
  __shared__ double s_tile[kRowChunk][kThreads];
  double *A = p.scratch + (int64_t)blockIdx.x * p.slot_stride;
  double *B = A + p.slot_stride / 2;
  const int nvecs = p.nvecs;
  const int nvc = (nvecs + VC - 1) / VC;
  for (;;) {
    int idx = next_matrix(p.counter, &s_idx);
    if (idx >= p.nmats) break;
    const DevMatrix M = p.mats[p.order[idx]];
    const double *qm = p.q_in + (int64_t)(2 * M.m + M.odd) * p.q_mstride;
    const double *level0 = M.nlevels > 0 ? A : qm;
    const int64_t l0s = M.nlevels > 0 ? nvecs : p.q_rstride;  // row stride of level0
    const int64_t arow0 = alm_row0(M, p.lmax);

    // ---- interpolation levels, leaf side to root side ----
    for (int t = M.nlevels - 1; t >= 0; --t) {
      const DevLevel L = p.levels[M.level_begin + t];
      double *upper = (t & 1) ? B : A;
      const double *lower = (t == M.nlevels - 1) ? qm : ((t & 1) ? A : B);
      const int64_t lws = (t == M.nlevels - 1) ? p.q_rstride : nvecs;  // row stride of lower
      const int32_t *um = p.i32 + L.upper_map;
      const int n_items = L.upper_rows * nvc;
      for (int it = threadIdx.x; it < n_items; it += blockDim.x) {
        const int row = it % L.upper_rows, v0 = (it / L.upper_rows) * VC;
        const int nv = min(VC, nvecs - v0);
        const DevPair P = p.pairs[um[2 * row]];
        const int sg = um[2 * row + 1];
        const bool isB = sg < 0;
        const int s = isB ? -(1 + sg) : sg;
        const int k = isB ? P.kB : P.kT;
        const int32_t *perm = p.i32 + (isB ? P.permB : P.permT);
        const double *w = p.f64 + (isB ? P.ipB : P.ipT) + s;
        auto lrow = [&](int zz) -> int64_t {
          return zz < P.n_left ? (int64_t)(P.out_left + zz) : (int64_t)(P.out_right + zz - P.n_left);
        };
        double acc[VC], x[VC];
        load_vec<VC>(acc, lower + lrow(perm[s]) * lws + v0, nv);
        const int nmk = P.n - k;
        for (int c = 0; c < nmk; ++c) {
          const double wc = w[(int64_t)c * k];
          load_vec<VC>(x, lower + lrow(perm[k + c]) * lws + v0, nv);
#pragma unroll
          for (int v = 0; v < VC; ++v) acc[v] += wc * x[v];
        }
        double *out = upper + (int64_t)row * nvecs + v0;
#pragma unroll
        for (int v = 0; v < VC; ++v)
          if (v < nv) out[v] = acc[v];
      }
      __syncthreads();
    }

    // ---- zero this matrix's alm rows, then accumulate D blocks ----
    for (int it = threadIdx.x; it < M.nk * nvecs; it += blockDim.x) {
      const int kk = it / nvecs, v = it % nvecs;
      p.alm_out[(arow0 + 2 * (int64_t)kk) * nvecs + v] = 0.0;
    }
    __syncthreads();
    const int32_t *rmap = p.i32 + M.root_map;
    for (int b = M.dblock_begin; b < M.dblock_end; ++b) {
      const DevDBlock D = p.dblocks[b];
      if (D.nrows == 0 || D.ncols == 0) continue;
      for (int c0 = 0; c0 < D.ncols; c0 += kThreads) {
        // this thread's column
        const int c = c0 + threadIdx.x;
        const bool have = c < D.ncols;
        DevStrip S{};
        int cl = 0;
        double x2 = 0, pp = 0, pc = 0;
        if (have) {
          const int row = D.out_row + c;
          S = p.strips[rmap[2 * row]];
          cl = rmap[2 * row + 1];
          if (S.kind == 1) {
            const int nx = S.cstop - S.cstart;
            const double *base = p.f64 + S.data;
            x2 = base[cl];
            pp = base[nx + cl];
            pc = base[2 * nx + cl];
          }
        }
        const int gcols = min(kThreads, D.ncols - c0);
        for (int k0 = 0; k0 < D.nrows; k0 += kRowChunk) {
          // recurrence tile: rows k0 .. k0 + kRowChunk - 1 of this column
#pragma unroll 1
          for (int r = 0; r < kRowChunk; ++r) {
            const int kk = k0 + r;
            double val = 0.0;
            if (have && kk < D.nrows && kk >= S.rstart) {
              const int kl = kk - S.rstart;
              if (S.kind == 0) {
                val = p.f64[S.data + (int64_t)cl * (D.nrows - S.rstart) + kl];
              } else if (kl == 0) {
                val = pp;
              } else if (kl == 1) {
                val = pc;
              } else {
                const double *ab = p.f64 + D.aux + 3 * (int64_t)(kk - 2);
                const double nv2 = (x2 + ab[0]) * ab[1] * pc + ab[2] * pp;
                pp = pc;
                pc = nv2;
                val = nv2;
              }
            }
            s_tile[r][threadIdx.x] = val;
          }
          __syncthreads();
          // tile product: out[r][v] = sum_c tile[r][c] * X[c][v]
          const int nrow = min(kRowChunk, D.nrows - k0);
          const int nout = nrow * nvecs;
          int tpo = kThreads / max(nout, 1);   // threads per output, power of two <= 32
          tpo = tpo >= 32 ? 32 : tpo >= 16 ? 16 : tpo >= 8 ? 8 : tpo >= 4 ? 4 : tpo >= 2 ? 2 : 1;
          const int per_pass = kThreads / tpo;
          const double *X = level0 + (int64_t)(D.out_row + c0) * l0s;
          for (int o0 = 0; o0 < nout; o0 += per_pass) {
            const int o = o0 + threadIdx.x / tpo, lane = threadIdx.x % tpo;
            double sum = 0.0;
            const int r = o / nvecs, v = o % nvecs;
            if (o < nout)
              for (int cc = lane; cc < gcols; cc += tpo) sum += s_tile[r][cc] * X[(int64_t)cc * l0s + v];
            for (int off = tpo / 2; off > 0; off >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, off);
            if (o < nout && lane == 0) {
              double *dst = p.alm_out + (arow0 + 2 * (int64_t)(D.row_start + k0 + r)) * nvecs + v;
              *dst += sum;
            }
          }
          __syncthreads();
        }
      }
    }
  }
}

template <int VC>
cudaError_t launch_vc(bool forward, const LegendreParams &prm, int grid, cudaStream_t st) {
  if (forward) {
    k_alm2map_legendre<VC><<<grid, kThreads, 0, st>>>(prm);
  } else {
    k_map2alm_legendre<VC><<<grid, kThreads, 0, st>>>(prm);
  }
  return cudaGetLastError();
}

}  // namespace

int legendre_threads() { return kThreads; }

// Loads the alm2map kernels' module now (module loading is lazy by default:
// the first launch would otherwise load it, and loading allocates device
// memory for the code).
cudaError_t legendre_preload() {
  cudaFuncAttributes a;
  cudaError_t e = cudaFuncGetAttributes(&a, k_alm2map_legendre<2>);
  if (e == cudaSuccess) e = cudaFuncGetAttributes(&a, k_alm2map_legendre<4>);
  if (e == cudaSuccess) e = cudaFuncGetAttributes(&a, k_alm2map_legendre<8>);
  return e;
}

cudaError_t launch_legendre(bool alm2map, const LegendreParams &prm, int grid, cudaStream_t st) {
  if (prm.nvecs <= 2) return launch_vc<2>(alm2map, prm, grid, st);
  if (prm.nvecs <= 4) return launch_vc<4>(alm2map, prm, grid, st);
  return launch_vc<8>(alm2map, prm, grid, st);
}

}  // namespace wm
