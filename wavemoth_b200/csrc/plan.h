// Device-side program of a butterfly-compressed Legendre transform.
//
// The host compiles every (m, parity) matrix of a rev1 resource file into
// flat, level-major tables that live in one device arena:
//
//   DevMatrix  one per (m, parity): its residual blocks and its levels
//   DevDBlock  one residual ("D") block of a forest root: rows
//              [row_start, row_start + nrows) of the matrix (row k <-> l =
//              m + parity + 2k) restricted to `ncols` skeleton columns, cut
//              into strips
//   DevStrip   columns [cstart, cstop) of a D block, rows [rstart, nrows):
//              dense values or (x^2, P0, P1) for the three-term recurrence
//   DevLevel   one tree depth: the interpolation pairs of every node at that
//              depth, mapping the blocks of the upper (root-side) buffer to
//              the blocks of the lower (leaf-side) buffer
//   DevPair    the (T, B) interpolation blocks of one node pair slot
//
// State buffers: the blocks of all nodes at one tree depth are stored
// back to back (heap order, then block order), `nvecs` doubles per row.  The
// leaf depth buffer is the Legendre output q itself (rows = rings), so the
// last level of alm2map writes q directly and the first level of map2alm
// reads q~ directly.
#pragma once
#include <stdint.h>

namespace wm {

struct DevStrip {
  int32_t rstart;   // first row (within the D block)
  int32_t cstart;   // first column (within the D block)
  int32_t cstop;
  int32_t kind;     // 0: dense (nrows - rstart) x (cstop - cstart), column-major; 1: recurrence
  int32_t dblock;   // owning residual block
  int32_t pad;
  int64_t data;     // f64 arena offset; recurrence: x2[nx], P0[nx], P1[nx]
};

struct DevDBlock {
  int32_t row_start;
  int32_t nrows;
  int32_t ncols;
  int32_t out_row;      // first row of this block in the depth-0 buffer
  int32_t strip_begin;
  int32_t strip_end;
  int64_t aux;          // f64 arena offset of 3*(nrows-2) recurrence coefficients
};

struct DevPair {
  int32_t kT, kB, n, n_left;
  int32_t inT, inB;            // rows of the skeleton blocks in the upper buffer
  int32_t out_left, out_right; // rows of the children's blocks in the lower buffer
  int64_t mapT, mapB;          // i32 arena, n entries: >= 0 interpolant column, < 0: -(1 + skeleton row)
  int64_t permT, permB;        // i32 arena, n entries: z positions of skeleton rows, then of columns
  int64_t ipT, ipB;            // f64 arena: k x (n-k) column-major
  int64_t ipT_t, ipB_t;        // f64 arena: (n-k) x k column-major (transposed copy)
};

struct DevLevel {
  int32_t pair_begin, pair_end;
  int32_t upper_rows, lower_rows;
  int64_t lower_map;     // i32 arena, 2 per lower row: (pair index, z = row within the pair's n)
  int64_t upper_map;     // i32 arena, 2 per upper row: (pair index, s >= 0 row of T, < 0: -(1+s) of B)
};

struct DevMatrix {
  int32_t m, odd, nk, ncols;
  int32_t nlevels;
  int32_t dblock_begin, dblock_end;
  int32_t level_begin;   // level_begin + t = tree depth t (0 = forest roots)
  int32_t root_rows;     // rows of the depth-0 buffer
  int32_t max_rows;      // rows of the largest intermediate buffer
  int64_t root_map;      // i32 arena, 2 per depth-0 row: (strip index, column within the strip)
  double cost;           // estimated work, for scheduling
  int64_t xrow;          // first row of this matrix in the X buffer (depth-1 matrices), else -1
  int32_t fast;          // 1: handled by the tensor-core path (depth <= 1)
  int32_t pad2;
};

// ---- tensor-core (DMMA) path for matrices of tree depth 0 or 1 ----
//
// A "row group" is the set of residual blocks that share one range of matrix
// rows: the single block of a depth-0 matrix, or the T (respectively B)
// blocks of all roots of a depth-1 matrix.  The residual products of a group
// are one GEMM with K = rows (alm2map) or K = the group's skeleton columns
// (map2alm) and a recurrence-generated operand.
struct DevGroup {
  int32_t matrix;     // index into the matrix table
  int32_t rs;         // first matrix row of the group
  int32_t nrows;
  int32_t ncols;      // skeleton columns of all the group's blocks
  int64_t cols;       // index of the group's first DevGCol
  int64_t seeds;      // index (in doubles) of the group's seeds: ncols x nchunks x 2
  int32_t nchunks;    // seed chunks of kSeedRows rows
  int32_t in_q;       // 1: the columns are rows of q (depth 0); 0: rows of the X buffer
};

struct DevGCol {
  int32_t row;        // row of this column in q or in the matrix's X buffer
  int32_t start;      // first active row (group coordinates); rows before it are zero
  int32_t boff;       // residual-block row offset: block row = group row - boff
  int32_t kind;       // 0: dense column, 1: recurrence
  int64_t data;       // dense: f64 offset of row `start`; recurrence: f64 offset of x^2
  int32_t nx;         // recurrence: stride from x^2 to P0 to P1
  int32_t pad;
  int64_t aux;        // f64 offset of the block's recurrence coefficients
};

struct DevTileA {     // alm2map residual unit: <= 64 consecutive group columns
  int32_t group, col0, ncols, kstart;
};

struct DevTileB {     // map2alm residual unit: <= kPushRows consecutive group rows
  int32_t group, row0, nrows, chunk;   // chunk: seed chunk of row0
};

struct DevRootUnit {  // depth-1 level unit: one root's interpolation pair
  int32_t matrix, pair;
};

constexpr int kPushRows = 32;   // rows of a map2alm residual unit (FP64 tensor-core path)
constexpr int kSeedRows = 16;   // spacing of the recurrence seeds (P at rows s, s + 1)

// ---- split-precision residual path (sliced int8 operands, tcgen05) ----
//
// The residual GEMMs of the row groups above, with both operands cut into
// kSplitSlices signed 7-bit slices under power-of-two scales (per skeleton
// column for alm2map, per matrix row for map2alm, per group and vector for
// the alm / X operand) and accumulated exactly in int32 on the tensor cores.
constexpr int kSplitSlices = 6;
constexpr int kSplitK = 64;       // K chunk (rows for alm2map, columns for map2alm)
constexpr int kSplitM = 128;      // M tile (columns for alm2map, rows for map2alm)
constexpr int kSplitN = 64;       // vectors per pass
constexpr int kSplitPlane = kSplitSlices * kSplitN * kSplitK;  // bytes of one operand chunk

struct DevSplitGroup {
  int64_t apl;        // first alm-operand chunk (alm2map): ceil(nrows / kSplitK) chunks
  int64_t xpl;        // first X-operand chunk (map2alm): ceil(ncols / kSplitK) chunks
  int64_t rowoff;     // first entry of the group's row scales
  int32_t nrchunks;
  int32_t ncchunks;
};

struct DevSplitTileA {  // alm2map: <= kSplitM columns of a group, K chunks from kc0
  int32_t group, col0, ncols, kc0;
};

struct DevSplitTileB {  // map2alm: <= kSplitM rows of a group, all its columns
  int32_t group, row0, nrows, pad;
};

// Split-precision level products of a depth-1 root (T, B) pair, W[z][s] the
// n x (kT + kB) interpolation matrix with the filter folded in:
//   alm2map   q[z] = sum_s W[z][s] X[s]     M = z (n), K = s (kT + kB)
//   map2alm   X[s] = sum_z W[z][s] q~[z]    M = s,     K = z
// W is sliced once per plan into A chunks laid out as shared memory wants
// them (kSplitSlices x kSplitM x kSplitK bytes each), per-row scales.
struct DevSplitRoot {
  int64_t a_a2m, a_m2a;     // first A chunk of each direction (M tiles x K chunks)
  int64_t b_a2m, b_m2a;     // first operand-B chunk (X over s, q~ over z)
  int64_t rs_a2m, rs_m2a;   // first row scale (n rows, kT + kB rows)
  int32_t nzc, nsc;         // chunks of 64 over z and over s
};

// Dense-recurrence plans: where the device Legendre seeds of column (m,
// parity, ring) go in the FP64 arena -- the value at row kstart + t, t <
// count, at base + t stride (P0 and P1 of a recurrence strip: count 2,
// stride nx; a dense strip of nks rows: count nks, stride 1).
struct DevDenseFill {
  int64_t base;
  int32_t stride;
  int32_t count;
};

// Rows that no split tile writes, zeroed before the launch they belong to:
// (buffer << kZeroBufShift) | row, buffer 0 q, 1 X buffer, 2 alm.
constexpr int kZeroBufShift = 56;

struct DevSplitLevelTile {  // <= kSplitM rows (z or s) of one root unit
  int32_t unit, row0, nrows, pad;
};

// One M tile of a streamed split GEMM: every operand chunk is read from
// global memory (A chunks sliced once per plan, B planes sliced per call),
// so residual and level products of both directions share one kernel.
// Output row r of the tile goes to row rows[tile * kSplitM + r] of the
// destination buffer (-1: none), scaled by 1 / scale of that tile row
// (entry scale_idx[tile * kSplitM + r] of the launch's scale table).
struct DevStreamTile {
  int64_t a;       // first A chunk (kSplitSlices x kSplitM x kSplitK bytes each)
  int64_t b;       // first B plane (kSplitPlane bytes each)
  int32_t nk;      // K chunks (> 0)
  int32_t vs;      // vector-scale row: group, or ngroups + root unit
  int32_t buf;     // destination: 0 q, 1 X buffer, 2 alm
  int32_t pad;
};

// Per ring pair (ring number r from the equator).
struct DevRing {
  int32_t n;              // pixels in the ring
  int32_t phi_num;        // phi0 = pi * phi_num / phi_den
  int32_t phi_den;
  int32_t bluestein_m;    // 0: n/2 is a power of two; else the Bluestein convolution length
  int64_t off_north;      // first pixel of ring mid - r
  int64_t off_south;      // first pixel of ring mid + r (== off_north at the equator)
  int64_t filter;         // Bluestein: complex offset of the filter spectrum (bit-reversed)
  int64_t aux;            // Bluestein: complex offset of chirp[n/2] then root[n/2 + 1]
};

// One CTA of a ring kernel: ring pair `ring`, maps [map0, map0 + 2^lg), both
// hemispheres at once if `two` (else one after the other).
struct DevRingTask {
  int32_t ring;
  int32_t map0;
  int32_t lg;
  int32_t pad;   // two
};

// Device-resident error word (never trap: kernels record and return).
enum : int32_t {
  kStatusOk = 0,
  kStatusBadProgram = 1,   // a table entry out of range
  kStatusTimeout = 2,      // a bounded wait gave up
};

}  // namespace wm
