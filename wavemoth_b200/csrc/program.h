// Host-side container of a compiled device program (see plan.h).
#pragma once
#include <stdint.h>
#include <string>
#include <vector>

#include "plan.h"

namespace wm {

struct HostProgram {
  int nside = 0, lmax = 0, mmax = 0;
  // m-sharded plans: the matrices of m in [shard_m0, shard_m1) are this
  // plan's (shard_m1 < 0: all), and its q holds only those m (q_row)
  int32_t shard_m0 = 0, shard_m1 = -1;
  int32_t max_rows = 0;                 // largest intermediate buffer over all matrices
  std::vector<DevMatrix> mats;          // (m, odd) in file order: index 2m + odd
  std::vector<DevDBlock> dblocks;
  std::vector<DevStrip> strips;
  std::vector<DevLevel> levels;
  std::vector<DevPair> pairs;
  std::vector<double> f64;
  std::vector<int32_t> i32;
  std::vector<int64_t> element_count;   // header element_count per (2m + odd)
  // tensor-core path tables (see plan.h)
  std::vector<DevGroup> groups;
  std::vector<DevGCol> gcols;
  std::vector<DevTileA> tiles_a;
  std::vector<DevTileB> tiles_b;
  std::vector<DevRootUnit> roots;
  std::vector<int32_t> slow_mats;       // matrices left to the generic kernels
  int64_t nseeds = 0;                   // doubles of recurrence seeds
  int64_t xrows = 0;                    // rows of the X buffer
  int32_t max_root_k = 0;               // largest kT + kB of a depth-1 root
  int32_t max_root_n = 0;               // largest n of a depth-1 root
  // split-precision residual tables (see plan.h)
  std::vector<DevSplitGroup> sgroups;   // one per group
  std::vector<DevSplitTileA> stiles_a;
  std::vector<DevSplitTileB> stiles_b;
  int64_t split_chunks = 0;             // operand-B chunks of the largest use
  int64_t split_rows = 0;               // row scales (sum of group rows)
  std::vector<DevSplitRoot> sroots;     // one per root unit
  std::vector<DevSplitLevelTile> stiles_la, stiles_lm;  // alm2map / map2alm level tiles
  int64_t split_level_achunks = 0;      // A chunks of W, both directions
  int64_t split_level_rows = 0;         // row scales of W, both directions
  // streamed split GEMM launches (kStream* order): the tiles, and per tile
  // row its destination row and scale index (-1: padding row)
  std::vector<DevStreamTile> stream_tiles[4];
  std::vector<int32_t> stream_rows[4], stream_sidx[4];
  int64_t stream_res_achunks = 0;       // A chunks of sliced residual P, both directions
  // destination rows that no split tile writes (columns with no active row,
  // roots with no skeleton) and that must read as zero, per launch
  // (kStream* order); encoded kZeroBufShift-bit buffer (0 q, 1 X, 2 alm)
  // above the row index
  std::vector<int64_t> split_zero[4];
  // per ring pair: 1 + the largest m for which the ring's Legendre column
  // (either parity) has a value above the plan writer's inclusion threshold
  // 1e-30; the q rows of larger m hold at most 1e-30 |a|, and the synthesis
  // gather of an alm2map stops there (empty: no limit)
  std::vector<int32_t> ring_mend;
  // algorithmic work of one transform direction
  int64_t interp_elems = 0;      // sum of k (n - k) over interpolation blocks
  int64_t rec_elems = 0;         // recurrence-strip elements (rows x columns)
  int64_t dense_elems = 0;       // dense residual elements
  int64_t rec_columns = 0;       // columns of recurrence strips (x2, P0, P1 each)
  int64_t aux_values = 0;        // recurrence coefficients stored
};

// Row of q (rows of nvecs doubles) holding (m, parity, ring): ring-major, so
// that the q block of one ring pair -- every (m, parity) of it -- is one
// contiguous range (rows ring * 2 (mmax + 1) .. + 2 (mmax + 1)).
inline int64_t q_row(int mmax, int m, int odd, int64_t ring) {
  return (ring * (mmax + 1) + m) * 2 + odd;
}
inline int64_t q_row(const HostProgram &P, int m, int odd, int64_t ring) {
  if (P.shard_m1 < 0) return q_row(P.mmax, m, odd, ring);
  // a shard's q holds rows of its own m only: ring stride 2 (m1 - m0); the
  // row index keeps m itself, the buffer's origin is moved back by 2 m0 rows
  return (ring * (P.shard_m1 - P.shard_m0) + m) * 2 + odd;
}

// Streamed split GEMM launches.
enum : int { kStreamResA2M = 0, kStreamResM2A = 1, kStreamLevelA2M = 2, kStreamLevelM2A = 3 };

// Builds the tensor-core path tables for matrices of depth 0 and 1.
bool build_fast_path(HostProgram &P, std::string &err);

// One serialized butterfly matrix (the per-matrix layout of a rev1 file,
// starting at its header) compiled without its residual payloads: a single
// DevMatrix whose root buffer rows the caller provides.
bool compile_butterfly_tree(const char *data, size_t len, HostProgram &P, std::string &err);

// Ring-pair colatitude data of HEALPix (pair 0 = equator): z = cos(theta)
// of the northern ring of every pair (src/wavemoth.c:1199-1232 geometry).
std::vector<double> ring_pair_z(int nside);

// Dense-recurrence program (no butterfly): every (m, parity) a depth-0
// matrix with one block over all rings, column r starting at row
// kstart[(2m + parity) ni + r]; the stored seed values are left zero and
// listed in `fill` for the device (launch_dense_fill).
bool build_dense_program(int nside, int lmax, int mmax, const std::vector<int32_t> &kstart, HostProgram &P,
                         std::vector<DevDenseFill> &fill, std::string &err);

// Parses a rev1 file image.  nside_expect < 0 accepts any nside.
bool compile_resource(const char *data, size_t len, int nside_expect, int lmax_expect,
                      int mmax_expect, HostProgram &P, std::string &err);

}  // namespace wm
