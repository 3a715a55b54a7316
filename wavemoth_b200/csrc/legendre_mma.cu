// Tensor-core (FP64 DMMA, mma.sync m8n8k4) kernels of the butterfly Legendre
// step for matrices of tree depth 0 and 1 (see plan.h, build_fast_path).
//
// For one row group g (a set of residual blocks sharing rows [rs, rs+R)):
//   alm2map residual   X[c]  = sum_r P[r][c] a[r]      M = columns, K = rows
//   map2alm residual   a[r]  = sum_c P[r][c] X[c]      M = rows,    K = columns
// P[r][c] is produced by the three-term recurrence of column c
// (src/legendre_transform.c.in:680-716) into a shared-memory tile and
// consumed by DMMA fragments.  For a depth-1 root (T, B) pair:
//   alm2map level      q[z] = sum_s W_T[z][s] X_T[s] + sum_s W_B[z][s] X_B[s]
//   map2alm level      X_T[s] = sum_z W_T[z][s] q~[z]   (and B)
// where W[z][s] is the (n x k) matrix of one interpolation block with its
// filter folded in: row z is the unit vector e_s' if z is skeleton column s'
// (filter 0), else column c(z) of the interpolant (src/butterfly.c.in:222-235).
//
// Fragment layout of mma.m8n8k4 .f64 (lane = 4 g + t): A (8x4, row) element
// (g, t); B (4x8, col) element (t, g); C/D (8x8) elements (g, 2t) and (g, 2t+1).
//
// Every output element has one writer and a fixed summation order, so results
// are bitwise reproducible.  map2alm rows of one group are split into units
// of kPushRows rows that start from recurrence seeds stored every kSeedRows
// rows (computed once per plan by k_seeds), so no cross-CTA reduction is
// needed.
#include <cuda_runtime.h>
#include <stdint.h>

#include "kernels.h"
#include "plan.h"

namespace wm {

namespace {

constexpr int kThr = 256;        // 8 warps
constexpr int kKC = 32;          // alm2map residual: rows per K chunk
constexpr int kTileCols = 256;   // alm2map residual: columns per tile (32 M-tiles)
constexpr int kPushCols = 256;   // map2alm residual: columns per K chunk

__device__ __forceinline__ void dmma(double (&d)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

__device__ __forceinline__ int64_t alm_row0(const DevMatrix &M, int lmax) {
  return (int64_t)M.m * (2 * lmax - M.m + 3) / 2 + M.odd;
}

// Recurrence step for group row r (>= start + 2) of column C.
__device__ __forceinline__ double rec_step(const double *f64, const DevGCol &C, double x2, int r,
                                           double pc, double pp) {
  const double *ab = f64 + C.aux + 3 * (int64_t)(r - C.boff - 2);
  return (x2 + ab[0]) * ab[1] * pc + ab[2] * pp;
}

// W[z][s] of one interpolation block (k skeleton columns, n rows z).
__device__ __forceinline__ double w_elem(const int32_t *map, const double *ip_t, int n, int k, int z,
                                         int s) {
  if (z >= n || s >= k) return 0.0;
  const int mt = map[z];
  if (mt < 0) return (s == -mt - 1) ? 1.0 : 0.0;
  return ip_t[mt + (int64_t)s * (n - k)];
}

// ------------------------------------------------------------------------
// alm2map residual: one unit = <= 256 columns of one group, all rows.  Every
// thread generates one column of the recurrence tile; warp w owns M-tiles
// w, w+8, w+16, w+24 (columns 8 mt ..) for all NT vector tiles.  The next
// chunk of alm rows is prefetched into registers during the products.
// ------------------------------------------------------------------------
template <int NT>
__global__ void __launch_bounds__(kThr, 1) k_a2m_residual(FastParams p) {
  constexpr int VT = 8 * NT;
  constexpr int VP = VT + 8;              // padded row stride (conflict-free fragments)
  constexpr int CP = kTileCols + 8;
  constexpr int PF = (kKC * VT + kThr - 1) / kThr;   // prefetched alm values per thread
  extern __shared__ double a2m_smem[];
  double(*a_tile)[VP] = reinterpret_cast<double(*)[VP]>(a2m_smem);
  double(*p_tile)[CP] = reinterpret_cast<double(*)[CP]>(a2m_smem + kKC * VP);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g4 = lane >> 2, t4 = lane & 3;
  for (int unit = blockIdx.x; unit < p.ntiles_a; unit += gridDim.x) {
    const DevTileA T = p.tiles_a[unit];
    const DevGroup G = p.groups[T.group];
    const DevMatrix M = p.mats[G.matrix];
    const int64_t arow0 = alm_row0(M, p.lmax);
    const int c = threadIdx.x;
    const bool gen = c < T.ncols;
    DevGCol C{};
    double x2 = 0.0, pp = 0.0, pc = 0.0;
    if (gen) {
      C = p.gcols[G.cols + T.col0 + c];
      if (C.kind == 1 && C.start < G.nrows) {
        x2 = p.f64[C.data];
        pp = p.f64[C.data + C.nx];
        pc = p.f64[C.data + 2 * C.nx];
      }
    }
    const int nmt = (T.ncols + 7) / 8;
    for (int v0 = 0; v0 < p.nvecs; v0 += VT) {
      const int vn = min(VT, p.nvecs - v0);
      double acc[4][NT][2];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int nt = 0; nt < NT; ++nt) acc[i][nt][0] = acc[i][nt][1] = 0.0;
      double gpp = pp, gpc = pc;
      double pf[PF];
      auto prefetch = [&](int r0) {
#pragma unroll
        for (int j = 0; j < PF; ++j) {
          const int idx = threadIdx.x + j * kThr;
          const int i = idx / VT, v = idx % VT, r = r0 + i;
          pf[j] = (idx < kKC * VT && r < G.nrows && v < vn)
                      ? p.alm_in[(arow0 + 2 * (int64_t)(G.rs + r)) * p.nvecs + v0 + v]
                      : 0.0;
        }
      };
      prefetch(T.kstart);
      for (int r0 = T.kstart; r0 < G.nrows; r0 += kKC) {
        __syncthreads();   // previous products done with both tiles
#pragma unroll
        for (int j = 0; j < PF; ++j) {
          const int idx = threadIdx.x + j * kThr;
          if (idx < kKC * VT) a_tile[idx / VT][idx % VT] = pf[j];
        }
        for (int i = 0; i < kKC; ++i) {
          const int r = r0 + i;
          double val = 0.0;
          if (gen && r >= C.start && r < G.nrows) {
            if (C.kind == 0) {
              val = p.f64[C.data + (r - C.start)];
            } else if (r == C.start) {
              val = gpp;
            } else if (r == C.start + 1) {
              val = gpc;
            } else {
              const double nv = rec_step(p.f64, C, x2, r, gpc, gpp);
              gpp = gpc;
              gpc = nv;
              val = nv;
            }
          }
          p_tile[i][c] = val;
        }
        __syncthreads();
        if (r0 + kKC < G.nrows) prefetch(r0 + kKC);
#pragma unroll 2
        for (int ks = 0; ks < kKC / 4; ++ks) {
          double b[NT];
#pragma unroll
          for (int nt = 0; nt < NT; ++nt) b[nt] = a_tile[4 * ks + t4][8 * nt + g4];
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            const int mt = warp + 8 * i;
            if (mt >= nmt) break;
            const double a = p_tile[4 * ks + t4][8 * mt + g4];
#pragma unroll
            for (int nt = 0; nt < NT; ++nt) dmma(acc[i][nt], a, b[nt]);
          }
        }
      }
      // epilogue: column 8 mt + g4, vectors 8 nt + 2 t4 + {0, 1}
      double *base = G.in_q ? p.q + (int64_t)(2 * M.m + M.odd) * p.q_mstride
                            : p.xbuf + M.xrow * p.nvecs;
      const int64_t rstride = G.in_q ? p.q_rstride : p.nvecs;
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int cc = 8 * (warp + 8 * i) + g4;
        if (cc >= T.ncols) continue;
        const DevGCol Co = p.gcols[G.cols + T.col0 + cc];
        double *dst = base + (int64_t)Co.row * rstride + v0;
#pragma unroll
        for (int nt = 0; nt < NT; ++nt) {
          const int v = 8 * nt + 2 * t4;
          if (v < vn) dst[v] = acc[i][nt][0];
          if (v + 1 < vn) dst[v + 1] = acc[i][nt][1];
        }
      }
      __syncthreads();
    }
  }
}

// ------------------------------------------------------------------------
// alm2map level: one unit = one depth-1 root; q rows = W_T X_T + W_B X_B.
// ------------------------------------------------------------------------
template <int NT>
__global__ void __launch_bounds__(kThr) k_a2m_level(FastParams p) {
  constexpr int VT = 8 * NT;
  constexpr int VP = VT + 8;
  extern __shared__ double xs[];  // (kT + kB rounded to 4) x VP
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g4 = lane >> 2, t4 = lane & 3;
  for (int unit = blockIdx.x; unit < p.nroots; unit += gridDim.x) {
    const DevRootUnit U = p.roots[unit];
    const DevMatrix M = p.mats[U.matrix];
    const DevPair P = p.pairs[U.pair];
    const int K = P.kT + P.kB, K4 = (K + 3) & ~3;
    const double *X = p.xbuf + M.xrow * p.nvecs;
    double *qm = p.q + (int64_t)(2 * M.m + M.odd) * p.q_mstride;
    const int32_t *mapT = p.i32 + P.mapT, *mapB = p.i32 + P.mapB;
    const double *ipT = p.f64 + P.ipT_t, *ipB = p.f64 + P.ipB_t;
    for (int v0 = 0; v0 < p.nvecs; v0 += VT) {
      const int vn = min(VT, p.nvecs - v0);
      __syncthreads();
      for (int idx = threadIdx.x; idx < K4 * VT; idx += kThr) {
        const int s = idx / VT, v = idx % VT;
        double val = 0.0;
        if (s < K && v < vn) {
          const int row = s < P.kT ? P.inT + s : P.inB + (s - P.kT);
          val = X[(int64_t)row * p.nvecs + v0 + v];
        }
        xs[s * VP + v] = val;
      }
      __syncthreads();
      for (int z0 = 0; z0 < P.n; z0 += 128) {
        double acc[2][NT][2];
#pragma unroll
        for (int i = 0; i < 2; ++i)
#pragma unroll
          for (int nt = 0; nt < NT; ++nt) acc[i][nt][0] = acc[i][nt][1] = 0.0;
        for (int ks = 0; ks < K4 / 4; ++ks) {
          const int s = 4 * ks + t4;
          double a[2];
#pragma unroll
          for (int i = 0; i < 2; ++i) {
            const int z = z0 + 16 * warp + 8 * i + g4;
            a[i] = s < P.kT ? w_elem(mapT, ipT, P.n, P.kT, z, s)
                            : w_elem(mapB, ipB, P.n, P.kB, z, s - P.kT);
          }
#pragma unroll
          for (int nt = 0; nt < NT; ++nt) {
            const double b = xs[s * VP + 8 * nt + g4];
            dmma(acc[0][nt], a[0], b);
            dmma(acc[1][nt], a[1], b);
          }
        }
#pragma unroll
        for (int i = 0; i < 2; ++i) {
          const int z = z0 + 16 * warp + 8 * i + g4;
          if (z >= P.n) continue;
          double *dst = qm + (int64_t)(P.out_left + z) * p.q_rstride + v0;
#pragma unroll
          for (int nt = 0; nt < NT; ++nt) {
            const int v = 8 * nt + 2 * t4;
            if (v < vn) dst[v] = acc[i][nt][0];
            if (v + 1 < vn) dst[v + 1] = acc[i][nt][1];
          }
        }
      }
    }
  }
}

// ------------------------------------------------------------------------
// map2alm level: one unit = one depth-1 root; X_T = W_T^T q~, X_B = W_B^T q~.
// ------------------------------------------------------------------------
template <int NT>
__global__ void __launch_bounds__(kThr) k_m2a_level(FastParams p) {
  constexpr int VT = 8 * NT;
  constexpr int VP = VT + 8;
  extern __shared__ double qs[];  // (n rounded to 4) x VP
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g4 = lane >> 2, t4 = lane & 3;
  for (int unit = blockIdx.x; unit < p.nroots; unit += gridDim.x) {
    const DevRootUnit U = p.roots[unit];
    const DevMatrix M = p.mats[U.matrix];
    const DevPair P = p.pairs[U.pair];
    const int n4 = (P.n + 3) & ~3;
    const double *qm = p.q_in + (int64_t)(2 * M.m + M.odd) * p.q_mstride;
    double *X = p.xbuf + M.xrow * p.nvecs;
    const int mtT = (P.kT + 7) / 8, mtB = (P.kB + 7) / 8, mtiles = mtT + mtB;
    for (int v0 = 0; v0 < p.nvecs; v0 += VT) {
      const int vn = min(VT, p.nvecs - v0);
      __syncthreads();
      for (int idx = threadIdx.x; idx < n4 * VT; idx += kThr) {
        const int z = idx / VT, v = idx % VT;
        double val = 0.0;
        if (z < P.n && v < vn) val = qm[(int64_t)(P.out_left + z) * p.q_rstride + v0 + v];
        qs[z * VP + v] = val;
      }
      __syncthreads();
      for (int mt = warp; mt < mtiles; mt += kThr / 32) {
        const bool isB = mt >= mtT;
        const int k = isB ? P.kB : P.kT;
        const int s = (isB ? mt - mtT : mt) * 8 + g4;
        const int32_t *map = p.i32 + (isB ? P.mapB : P.mapT);
        const double *ipt = p.f64 + (isB ? P.ipB_t : P.ipT_t);
        double acc[NT][2];
#pragma unroll
        for (int nt = 0; nt < NT; ++nt) acc[nt][0] = acc[nt][1] = 0.0;
        for (int ks = 0; ks < n4 / 4; ++ks) {
          const int z = 4 * ks + t4;
          const double a = w_elem(map, ipt, P.n, k, z, s);
#pragma unroll
          for (int nt = 0; nt < NT; ++nt) dmma(acc[nt], a, qs[(4 * ks + t4) * VP + 8 * nt + g4]);
        }
        if (s < k) {
          double *dst = X + (int64_t)((isB ? P.inB : P.inT) + s) * p.nvecs + v0;
#pragma unroll
          for (int nt = 0; nt < NT; ++nt) {
            const int v = 8 * nt + 2 * t4;
            if (v < vn) dst[v] = acc[nt][0];
            if (v + 1 < vn) dst[v + 1] = acc[nt][1];
          }
        }
      }
    }
  }
}

// ------------------------------------------------------------------------
// map2alm residual: one unit = kPushRows rows of one group, all its columns.
// ------------------------------------------------------------------------
template <int NT>
__global__ void __launch_bounds__(kThr, 1) k_m2a_residual(FastParams p) {
  constexpr int VT = 8 * NT;
  constexpr int VP = VT + 8;
  constexpr int PP = kPushCols + 4;       // rows of 8 fragments hit all banks
  constexpr int TILES = 4 * NT;           // 4 M-tiles (32 rows) x NT N-tiles
  constexpr int PER_WARP = (TILES + 7) / 8;
  extern __shared__ double push_smem[];
  double(*p_tile)[PP] = reinterpret_cast<double(*)[PP]>(push_smem);
  double(*x_tile)[VP] = reinterpret_cast<double(*)[VP]>(push_smem + kPushRows * PP);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g4 = lane >> 2, t4 = lane & 3;
  for (int unit = blockIdx.x; unit < p.ntiles_b; unit += gridDim.x) {
    const DevTileB T = p.tiles_b[unit];
    const DevGroup G = p.groups[T.group];
    const DevMatrix M = p.mats[G.matrix];
    const int64_t arow0 = alm_row0(M, p.lmax);
    const double *Xb = G.in_q ? p.q_in + (int64_t)(2 * M.m + M.odd) * p.q_mstride
                              : p.xbuf + M.xrow * p.nvecs;
    const int64_t rstride = G.in_q ? p.q_rstride : p.nvecs;
    for (int v0 = 0; v0 < p.nvecs; v0 += VT) {
      const int vn = min(VT, p.nvecs - v0);
      double acc[PER_WARP][2];
#pragma unroll
      for (int j = 0; j < PER_WARP; ++j) acc[j][0] = acc[j][1] = 0.0;
      for (int c0 = 0; c0 < G.ncols; c0 += kPushCols) {
        const int nc = min(kPushCols, G.ncols - c0);
        __syncthreads();
        // recurrence tile: thread c generates column c0 + c for the unit's rows
        {
          const int c = threadIdx.x;
          if (c < nc) {
            const DevGCol C = p.gcols[G.cols + c0 + c];
            const double *seed = p.seeds + G.seeds + ((int64_t)(c0 + c) * G.nchunks + T.chunk) * 2;
            const int s0 = max(T.row0, C.start);
            double gpp = 0.0, gpc = 0.0, x2 = 0.0;
            if (C.kind == 1 && s0 < G.nrows) {
              gpp = seed[0];
              gpc = seed[1];
              x2 = p.f64[C.data];
            }
            for (int i = 0; i < kPushRows; ++i) {
              const int r = T.row0 + i;
              double val = 0.0;
              if (i < T.nrows && r >= C.start) {
                if (C.kind == 0) {
                  val = p.f64[C.data + (r - C.start)];
                } else if (r == s0) {
                  val = gpp;
                } else if (r == s0 + 1) {
                  val = gpc;
                } else {
                  const double nv = rec_step(p.f64, C, x2, r, gpc, gpp);
                  gpp = gpc;
                  gpc = nv;
                  val = nv;
                }
              }
              p_tile[i][c] = val;
            }
          } else {
            for (int i = 0; i < kPushRows; ++i) p_tile[i][c] = 0.0;
          }
        }
        {
          // X rows of the chunk, warp-cooperative: LPC lanes per row, two
          // vectors (16 bytes) per lane, so one load instruction covers
          // whole rows
          constexpr int LPC = VT / 2, RPI = 32 / LPC;
          for (int cb = warp * RPI; cb < kPushCols; cb += 8 * RPI) {
            const int c = cb + lane / LPC, v = 2 * (lane % LPC);
            double2 val = make_double2(0.0, 0.0);
            if (c < nc && v < vn)
              val = *reinterpret_cast<const double2 *>(
                  Xb + (int64_t)p.gcols[G.cols + c0 + c].row * rstride + v0 + v);
            *reinterpret_cast<double2 *>(&x_tile[c][v]) = val;
          }
        }
        __syncthreads();
#pragma unroll
        for (int j = 0; j < PER_WARP; ++j) {
          const int t = warp + 8 * j;
          if (t >= TILES) break;
          const int mt = t & 3, nt = t >> 2;
#pragma unroll 4
          for (int ks = 0; ks < kPushCols / 4; ++ks)
            dmma(acc[j], p_tile[8 * mt + g4][4 * ks + t4], x_tile[4 * ks + t4][8 * nt + g4]);
        }
      }
#pragma unroll
      for (int j = 0; j < PER_WARP; ++j) {
        const int t = warp + 8 * j;
        if (t >= TILES) break;
        const int mt = t & 3, nt = t >> 2;
        const int i = 8 * mt + g4;
        if (i >= T.nrows) continue;
        double *dst = p.alm_out + (arow0 + 2 * (int64_t)(G.rs + T.row0 + i)) * p.nvecs + v0;
        const int v = 8 * nt + 2 * t4;
        if (v < vn) dst[v] = acc[j][0];
        if (v + 1 < vn) dst[v + 1] = acc[j][1];
      }
    }
  }
}

// ------------------------------------------------------------------------
// Seeds: P at rows (s, s + 1), s = max(chunk start, column start), for every
// recurrence column and row chunk of its group.
// ------------------------------------------------------------------------
__global__ void k_seeds(FastParams p) {
  const int64_t gc = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (gc >= p.ngcols) return;
  // locate the group (binary search over group column offsets)
  int lo = 0, hi = p.ngroups - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) / 2;
    if (p.groups[mid].cols <= gc) lo = mid; else hi = mid - 1;
  }
  const DevGroup G = p.groups[lo];
  const int c = (int)(gc - G.cols);
  const DevGCol C = p.gcols[gc];
  double *seed = p.seeds_out + G.seeds + (int64_t)c * G.nchunks * 2;
  for (int j = 0; j < G.nchunks; ++j) {
    seed[2 * j] = 0.0;
    seed[2 * j + 1] = 0.0;
  }
  if (C.kind != 1 || C.start >= G.nrows) return;
  const double x2 = p.f64[C.data];
  double a = p.f64[C.data + C.nx], b = p.f64[C.data + 2 * C.nx];  // P[row], P[row + 1]
  int row = C.start;
  for (int j = 0; j < G.nchunks; ++j) {
    const int target = max(j * kSeedRows, C.start);
    if (target >= G.nrows) break;
    while (row < target) {
      // P[row + 2] exists only inside the group's rows
      const double nv = (row + 2 < G.nrows) ? rec_step(p.f64, C, x2, row + 2, b, a) : 0.0;
      a = b;
      b = nv;
      ++row;
    }
    seed[2 * j] = a;
    seed[2 * j + 1] = b;
  }
}

template <int NT>
cudaError_t launch_nt(int which, const FastParams &prm, int grid, size_t smem, cudaStream_t st) {
  switch (which) {
    case 0: {
      const size_t sm = (size_t)(kKC * (8 * NT + 8) + kKC * (kTileCols + 8)) * sizeof(double);
      cudaError_t e = cudaFuncSetAttribute(k_a2m_residual<NT>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
      if (e != cudaSuccess) return e;
      k_a2m_residual<NT><<<grid, kThr, sm, st>>>(prm);
      break;
    }
    case 1: {
      cudaError_t e = cudaFuncSetAttribute(k_a2m_level<NT>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e != cudaSuccess) return e;
      k_a2m_level<NT><<<grid, kThr, smem, st>>>(prm);
      break;
    }
    case 2: {
      cudaError_t e = cudaFuncSetAttribute(k_m2a_level<NT>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e != cudaSuccess) return e;
      k_m2a_level<NT><<<grid, kThr, smem, st>>>(prm);
      break;
    }
    case 3: {
      const size_t sm = (size_t)(kPushRows * (kPushCols + 4) + kPushCols * (8 * NT + 8)) * sizeof(double);
      cudaError_t e = cudaFuncSetAttribute(k_m2a_residual<NT>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
      if (e != cudaSuccess) return e;
      k_m2a_residual<NT><<<grid, kThr, sm, st>>>(prm);
      break;
    }
  }
  return cudaGetLastError();
}

}  // namespace

int fast_vector_tiles(int nvecs) {
  // N-tiles of 8 vectors per pass: the smallest power of two covering
  // nvecs, at most 8 (64 vectors per pass)
  int nt = 1;
  while (nt < 8 && 8 * nt < nvecs) nt *= 2;
  return nt;
}

cudaError_t launch_fast(int which, const FastParams &prm, int grid, cudaStream_t st) {
  const int NT = fast_vector_tiles(prm.nvecs);
  const int VP = 8 * NT + 8;
  size_t smem = 0;
  if (which == 1) smem = (size_t)((prm.max_root_k + 3) & ~3) * VP * sizeof(double);
  if (which == 2) smem = (size_t)((prm.max_root_n + 3) & ~3) * VP * sizeof(double);
  if (which == 1 || which == 2) smem = smem < 16 ? 16 : smem;
  switch (NT) {
    case 1: return launch_nt<1>(which, prm, grid, smem, st);
    case 2: return launch_nt<2>(which, prm, grid, smem, st);
    case 4: return launch_nt<4>(which, prm, grid, smem, st);
    default: return launch_nt<8>(which, prm, grid, smem, st);
  }
}

cudaError_t launch_seeds(const FastParams &prm, cudaStream_t st) {
  if (prm.ngcols == 0) return cudaSuccess;
  const int block = 128;
  const int64_t grid = (prm.ngcols + block - 1) / block;
  k_seeds<<<(unsigned)grid, block, 0, st>>>(prm);
  return cudaGetLastError();
}

}  // namespace wm
