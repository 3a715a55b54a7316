// rev1 resource file -> flat device program (plan.h).
//
// The rev1 layout read here is the reference's (src/wavemoth.c:203-264 for
// the file header, src/butterfly.c.in:284-445 and src/butterfly.h.in:8-88 for
// one matrix, src/wavemoth.c:958-1009 for a residual payload).  Unlike the
// reference reader, every offset, count and size is range-checked against
// the file so that a truncated or corrupt file yields an error message, not
// a crash.
#include <stdint.h>
#include <string.h>
#include <algorithm>
#include <string>
#include <vector>

#include "legendre.cuh"
#include "plan.h"
#include "program.h"

namespace wm {

namespace {

struct Reader {
  const char *base;
  size_t len;
  std::string *err;
  bool ok = true;

  bool fail(const std::string &msg) {
    if (ok) *err = msg;
    ok = false;
    return false;
  }
  bool check(size_t off, size_t n, const char *what) {
    if (off > len || n > len - off) return fail(std::string("resource file truncated: ") + what);
    return true;
  }
  template <class T>
  T get(size_t off, const char *what) {
    T v{};
    if (check(off, sizeof(T), what)) memcpy(&v, base + off, sizeof(T));
    return v;
  }
};

inline size_t pad16(size_t off) { return (off + 15) & ~size_t(15); }

struct NodeInfo {
  bool present = false;
  int32_t nblocks = 0;           // 0 for a leaf
  std::vector<int32_t> heights;  // leaf: {n}
  size_t data = 0;               // file offset just after the heights
};

size_t append_f64(std::vector<double> &arena, const char *src, size_t n) {
  size_t off = (arena.size() + 3) & ~size_t(3);
  arena.resize(off + n);
  if (n) memcpy(arena.data() + off, src, n * sizeof(double));
  return off;
}

size_t append_i32(std::vector<int32_t> &arena, const std::vector<int32_t> &v) {
  size_t off = (arena.size() + 3) & ~size_t(3);
  arena.resize(off + v.size());
  std::copy(v.begin(), v.end(), arena.begin() + off);
  return off;
}

bool compile_matrix(Reader &R, size_t start, int m, int odd, int nk_expect, int ncols_expect,
                    HostProgram &P, bool tree_only = false) {
  if (start % 16 != 0) return R.fail("matrix data not 16-byte aligned");
  int32_t nrows = R.get<int32_t>(start + 0, "matrix header");
  int32_t ncols = R.get<int32_t>(start + 4, "matrix header");
  int64_t element_count = R.get<int64_t>(start + 16, "matrix header");
  int32_t nroots = R.get<int32_t>(start + 24, "matrix header");
  int32_t heap_size = R.get<int32_t>(start + 28, "matrix header");
  int32_t heap_first = R.get<int32_t>(start + 32, "matrix header");
  if (!R.ok) return false;
  char buf[256];
  if (ncols != ncols_expect || nrows != nk_expect) {
    snprintf(buf, sizeof buf, "matrix m=%d odd=%d has shape %dx%d, expected %dx%d", m, odd, nrows,
             ncols, nk_expect, ncols_expect);
    return R.fail(buf);
  }
  if (nroots <= 0 || heap_size < nroots || heap_first < 1 || heap_first > (1 << 24) ||
      heap_size > (1 << 24))
    return R.fail("matrix header has an invalid forest/heap description");
  size_t table = start + 40;
  std::vector<int64_t> res_off(nroots), heap_off(heap_size);
  for (int i = 0; i < nroots; ++i) res_off[i] = R.get<int64_t>(table + 8 * i, "residual table");
  for (int i = 0; i < heap_size; ++i)
    heap_off[i] = R.get<int64_t>(table + 8 * (nroots + i), "heap table");
  if (!R.ok) return false;

  auto node = [&](int64_t pos, NodeInfo &ni) -> bool {
    int64_t idx = pos - heap_first;
    if (idx < 0 || idx >= heap_size) return R.fail("heap position out of range");
    if (heap_off[idx] <= 0) return R.fail("missing heap node");
    size_t off = start + (size_t)heap_off[idx];
    ni.present = true;
    ni.nblocks = R.get<int32_t>(off, "node");
    if (ni.nblocks < 0 || ni.nblocks > (1 << 20)) return R.fail("invalid node block count");
    if (ni.nblocks == 0) {
      ni.heights = {R.get<int32_t>(off + 4, "leaf node")};
      ni.data = off + 8;
    } else {
      ni.heights.resize(ni.nblocks);
      if (!R.check(off + 4, 4 * (size_t)ni.nblocks, "node heights")) return false;
      memcpy(ni.heights.data(), R.base + off + 4, 4 * (size_t)ni.nblocks);
      ni.data = off + 4 + 4 * (size_t)ni.nblocks;
    }
    for (int32_t h : ni.heights)
      if (h < 0 || h > (1 << 24)) return R.fail("invalid block height");
    return R.ok;
  };

  // depth of the forest (all roots of a complete tree have the same depth)
  int depth = 0;
  {
    int64_t p = heap_first;
    NodeInfo ni;
    for (;;) {
      if (!node(p, ni)) return false;
      if (ni.nblocks == 0) break;
      ++depth;
      p *= 2;
      if (depth > 30) return R.fail("tree too deep");
    }
  }
  // nodes per depth, and row offsets of every block in that depth's buffer
  std::vector<std::vector<NodeInfo>> nodes(depth + 1);
  std::vector<std::vector<std::vector<int32_t>>> offs(depth + 1);
  std::vector<int32_t> rows_at(depth + 1, 0);
  for (int d = 0; d <= depth; ++d) {
    int64_t p0 = (int64_t)heap_first << d, p1 = ((int64_t)heap_first + nroots) << d;
    nodes[d].resize(p1 - p0);
    offs[d].resize(p1 - p0);
    int64_t row = 0;
    for (int64_t p = p0; p < p1; ++p) {
      NodeInfo &ni = nodes[d][p - p0];
      if (!node(p, ni)) return false;
      if ((d < depth) != (ni.nblocks > 0)) return R.fail("butterfly tree is not complete");
      for (int32_t h : ni.heights) {
        offs[d][p - p0].push_back((int32_t)row);
        row += h;
      }
      if (row > (1 << 28)) return R.fail("butterfly buffer too large");
    }
    rows_at[d] = (int32_t)row;
  }
  if (rows_at[depth] != ncols) return R.fail("leaf widths do not add up to the column count");

  DevMatrix M{};
  M.m = m;
  M.odd = odd;
  M.nk = nrows;
  M.ncols = ncols;
  M.nlevels = depth;
  M.dblock_begin = (int32_t)P.dblocks.size();
  M.level_begin = (int32_t)P.levels.size();
  M.root_rows = rows_at[0];
  M.max_rows = 0;
  for (int d = 0; d < depth; ++d) M.max_rows = std::max(M.max_rows, rows_at[d]);
  double cost = 0;

  // ---- interpolation levels ----
  for (int d = 0; d < depth; ++d) {
    DevLevel L{};
    L.pair_begin = (int32_t)P.pairs.size();
    L.upper_rows = rows_at[d];
    L.lower_rows = rows_at[d + 1];
    int64_t p0 = (int64_t)heap_first << d;
    for (size_t u = 0; u < nodes[d].size(); ++u) {
      const NodeInfo &ni = nodes[d][u];
      int64_t p = p0 + (int64_t)u;
      size_t cl = (size_t)(2 * p - ((int64_t)heap_first << (d + 1)));
      const NodeInfo &lc = nodes[d + 1][cl], &rc = nodes[d + 1][cl + 1];
      int npairs = ni.nblocks / 2;
      if (ni.nblocks % 2 != 0 || (int)lc.heights.size() != npairs ||
          (int)rc.heights.size() != npairs)
        return R.fail("children do not match the parent's block count");
      size_t off = ni.data;
      for (int i = 0; i < npairs; ++i) {
        DevPair pr{};
        pr.n_left = lc.heights[i];
        int32_t n = lc.heights[i] + rc.heights[i];
        pr.n = n;
        pr.out_left = offs[d + 1][cl][i];
        pr.out_right = offs[d + 1][cl + 1][i];
        for (int j = 0; j < 2; ++j) {
          int32_t k = ni.heights[2 * i + j];
          if (k > n) return R.fail("interpolation block has more rows than columns");
          if (!R.check(off, (size_t)n, "filter")) return false;
          const int8_t *filt = (const int8_t *)(R.base + off);
          std::vector<int32_t> map(n), perm(n);
          int zeros = 0, ones = 0;
          for (int z = 0; z < n; ++z)
            if (filt[z] == 0) ++zeros;
            else if (filt[z] == 1) ++ones;
            else return R.fail("filter entry not 0/1");
          if (zeros != k) return R.fail("filter does not select k skeleton columns");
          int s = 0, c = 0;
          for (int z = 0; z < n; ++z) {
            if (filt[z] == 0) { map[z] = -(1 + s); perm[s] = z; ++s; }
            else { map[z] = c; perm[k + c] = z; ++c; }
          }
          off = pad16(off + n);
          size_t nel = (size_t)k * (size_t)(n - k);
          if (!R.check(off, 8 * nel, "interpolant")) return false;
          const double *ip = (const double *)(R.base + off);
          off += 8 * nel;
          size_t ipo = append_f64(P.f64, (const char *)ip, nel);
          // transposed copy: (n-k) x k column-major
          std::vector<double> tr(nel);
          for (int c2 = 0; c2 < n - k; ++c2)
            for (int s2 = 0; s2 < k; ++s2) tr[c2 + (size_t)s2 * (n - k)] = ip[s2 + (size_t)c2 * k];
          size_t ipt = append_f64(P.f64, (const char *)tr.data(), nel);
          P.interp_elems += (int64_t)nel;
          size_t mo = append_i32(P.i32, map), po = append_i32(P.i32, perm);
          if (j == 0) {
            pr.kT = k; pr.inT = offs[d][u][2 * i]; pr.mapT = mo; pr.permT = po;
            pr.ipT = ipo; pr.ipT_t = ipt;
          } else {
            pr.kB = k; pr.inB = offs[d][u][2 * i + 1]; pr.mapB = mo; pr.permB = po;
            pr.ipB = ipo; pr.ipB_t = ipt;
          }
          cost += (double)nel + n;
        }
        P.pairs.push_back(pr);
      }
    }
    L.pair_end = (int32_t)P.pairs.size();
    std::vector<int32_t> lower(2 * (size_t)L.lower_rows, -1), upper(2 * (size_t)L.upper_rows, -1);
    for (int32_t pi = L.pair_begin; pi < L.pair_end; ++pi) {
      const DevPair &pr = P.pairs[pi];
      for (int32_t z = 0; z < pr.n; ++z) {
        int32_t row = z < pr.n_left ? pr.out_left + z : pr.out_right + (z - pr.n_left);
        if (row < 0 || row >= L.lower_rows || lower[2 * row] != -1)
          return R.fail("interpolation pairs do not tile the lower buffer");
        lower[2 * row] = pi;
        lower[2 * row + 1] = z;
      }
      for (int32_t s = 0; s < pr.kT + pr.kB; ++s) {
        int32_t row = s < pr.kT ? pr.inT + s : pr.inB + (s - pr.kT);
        if (row < 0 || row >= L.upper_rows || upper[2 * row] != -1)
          return R.fail("interpolation pairs do not tile the upper buffer");
        upper[2 * row] = pi;
        upper[2 * row + 1] = s < pr.kT ? s : -(1 + (s - pr.kT));
      }
    }
    for (size_t i = 0; i < lower.size(); i += 2)
      if (lower[i] == -1) {
        snprintf(buf, sizeof buf, "m=%d odd=%d depth %d: lower buffer row %zu of %d not produced",
                 m, odd, d, i / 2, L.lower_rows);
        return R.fail(buf);
      }
    for (size_t i = 0; i < upper.size(); i += 2)
      if (upper[i] == -1) {
        snprintf(buf, sizeof buf, "m=%d odd=%d depth %d: upper buffer row %zu of %d not consumed",
                 m, odd, d, i / 2, L.upper_rows);
        return R.fail(buf);
      }
    L.lower_map = (int64_t)append_i32(P.i32, lower);
    L.upper_map = (int64_t)append_i32(P.i32, upper);
    P.levels.push_back(L);
  }

  // ---- residual blocks of every forest root ----
  // (tree_only: the caller supplies the root rows; no payload is decoded)
  for (int r = 0; r < nroots && !tree_only; ++r) {
    const NodeInfo &root = nodes[0][r];
    int nb = (int)root.heights.size();
    if (res_off[r] <= 0) return R.fail("missing residual payload table");
    size_t toff = start + (size_t)res_off[r];
    int64_t n = R.get<int64_t>(toff, "residual payload table");
    if (!R.ok) return false;
    if (n != nb) return R.fail("residual payload count does not match the root");
    std::vector<int64_t> po(n + 1);
    for (int64_t j = 0; j <= n; ++j) po[j] = R.get<int64_t>(toff + 8 + 8 * j, "payload offsets");
    if (!R.ok) return false;
    for (int j = 0; j < nb; ++j) {
      DevDBlock D{};
      D.ncols = root.heights[j];
      D.out_row = offs[0][r][j];
      D.strip_begin = (int32_t)P.strips.size();
      D.aux = -1;
      size_t off = pad16(start + (size_t)po[j]);
      int64_t rs = R.get<int64_t>(off, "payload"), re = R.get<int64_t>(off + 8, "payload");
      if (!R.ok) return false;
      if (rs < 0 || re < rs || re > nrows) return R.fail("payload row range outside the matrix");
      off += 16;
      D.row_start = (int32_t)rs;
      D.nrows = (int32_t)(re - rs);
      int32_t nkb = D.nrows;
      if (nkb <= 4 || D.ncols == 0) {
        off = pad16(off);
        size_t nel = (size_t)nkb * D.ncols;
        if (!R.check(off, 8 * nel, "dense residual block")) return false;
        DevStrip S{0, 0, D.ncols, 0, (int32_t)P.dblocks.size(), 0,
                   (int64_t)append_f64(P.f64, R.base + off, nel)};
        P.dense_elems += (int64_t)nel;
        P.strips.push_back(S);
        cost += (double)nel;
      } else {
        int64_t nstrips = R.get<int64_t>(off, "strip count");
        off += 8;
        if (!R.ok) return false;
        if (nstrips <= 0 || nstrips > D.ncols + 1) return R.fail("invalid strip count");
        off = pad16(off);
        size_t naux = 3 * (size_t)(nkb - 2);
        if (!R.check(off, 8 * naux, "recurrence coefficients")) return false;
        D.aux = (int64_t)append_f64(P.f64, R.base + off, naux);
        P.aux_values += (int64_t)naux;
        off += 8 * naux;
        int32_t cstart = 0;
        for (int64_t s = 0; s < nstrips; ++s) {
          int64_t rstart = R.get<int64_t>(off, "strip"), cstop = R.get<int64_t>(off + 8, "strip");
          off += 16;
          if (!R.ok) return false;
          if (rstart < 0 || rstart > nkb || cstop < cstart || cstop > D.ncols)
            return R.fail("strip outside its residual block");
          int32_t nx = (int32_t)cstop - cstart, nks = nkb - (int32_t)rstart;
          DevStrip S{(int32_t)rstart, cstart, (int32_t)cstop, 0, (int32_t)P.dblocks.size(), 0, 0};
          if (nks <= 4) {
            off = pad16(off);
            size_t nel = (size_t)nks * nx;
            if (!R.check(off, 8 * nel, "dense strip")) return false;
            S.data = (int64_t)append_f64(P.f64, R.base + off, nel);
            off += 8 * nel;
            P.dense_elems += (int64_t)nel;
          } else {
            S.kind = 1;
            size_t o[3];
            for (int a = 0; a < 3; ++a) {
              off = pad16(off);
              if (!R.check(off, 8 * (size_t)nx, "recurrence strip")) return false;
              o[a] = off;
              off += 8 * (size_t)nx;
            }
            // keep x2, P0, P1 contiguous
            size_t base = (P.f64.size() + 3) & ~size_t(3);
            P.f64.resize(base + 3 * (size_t)nx);
            for (int a = 0; a < 3; ++a)
              memcpy(P.f64.data() + base + (size_t)a * nx, R.base + o[a], 8 * (size_t)nx);
            S.data = (int64_t)base;
            P.rec_elems += (int64_t)nks * nx;
            P.rec_columns += nx;
          }
          cost += (double)nks * nx * (S.kind ? 2.5 : 1.0);
          P.strips.push_back(S);
          cstart = (int32_t)cstop;
        }
        if (cstart != D.ncols) return R.fail("strips do not cover the residual block");
      }
      D.strip_end = (int32_t)P.strips.size();
      P.dblocks.push_back(D);
    }
  }
  M.dblock_end = (int32_t)P.dblocks.size();
  if (!tree_only) {
    std::vector<int32_t> rm(2 * (size_t)M.root_rows, -1);
    for (int32_t b = M.dblock_begin; b < M.dblock_end; ++b) {
      const DevDBlock &D = P.dblocks[b];
      for (int32_t s = D.strip_begin; s < D.strip_end; ++s) {
        const DevStrip &S = P.strips[s];
        for (int32_t c = S.cstart; c < S.cstop; ++c) {
          int32_t row = D.out_row + c;
          if (row < 0 || row >= M.root_rows || rm[2 * row] != -1)
            return R.fail("residual blocks do not tile the root buffer");
          rm[2 * row] = s;
          rm[2 * row + 1] = c - S.cstart;
        }
      }
    }
    for (int32_t v : rm)
      if (v == -1) return R.fail("root buffer row not produced by any residual block");
    M.root_map = (int64_t)append_i32(P.i32, rm);
  }
  M.cost = cost;
  P.element_count[2 * m + odd] = element_count;
  P.mats.push_back(M);
  return R.ok;
}

}  // namespace

bool compile_butterfly_tree(const char *data, size_t len, HostProgram &P, std::string &err) {
  Reader R{data, len, &err};
  const int32_t nrows = R.get<int32_t>(0, "matrix header"), ncols = R.get<int32_t>(4, "matrix header");
  if (!R.ok) return false;
  P = HostProgram{};
  P.element_count.assign(2, 0);
  if (!compile_matrix(R, 0, 0, 0, nrows, ncols, P, true)) return false;
  P.max_rows = P.mats[0].max_rows;
  return true;
}

std::vector<double> ring_pair_z(int nside) {
  std::vector<double> z(2 * (size_t)nside);
  const double ns = (double)nside;
  for (int r = 0; r < 2 * nside; ++r) {
    const double i = (double)(2 * nside - r);  // ring number counted from the north pole, from 1
    z[r] = i <= ns ? 1.0 - i * i / (3.0 * ns * ns) : 4.0 / 3.0 - 2.0 * i / (3.0 * ns);
  }
  return z;
}

bool build_dense_program(int nside, int lmax, int mmax, const std::vector<int32_t> &kstart, HostProgram &P,
                         std::vector<DevDenseFill> &fill, std::string &err) {
  const int ni = 2 * nside;
  if (nside <= 0 || lmax < 0 || mmax > lmax || kstart.size() != 2 * (size_t)(mmax + 1) * ni) {
    err = "dense program: inconsistent sizes";
    return false;
  }
  P = HostProgram{};
  P.nside = nside;
  P.lmax = lmax;
  P.mmax = mmax;
  P.element_count.assign(2 * (mmax + 1), 0);
  fill.assign(kstart.size(), DevDenseFill{0, 0, 0});
  const std::vector<double> z = ring_pair_z(nside);
  auto zeros = [&](size_t n) {
    const size_t off = (P.f64.size() + 3) & ~size_t(3);
    P.f64.resize(off + n, 0.0);
    return (int64_t)off;
  };
  for (int m = 0; m <= mmax; ++m) {
    for (int odd = 0; odd < 2; ++odd) {
      const int mi = 2 * m + odd;
      const int32_t nk = lmax - m - odd >= 0 ? (lmax - m - odd) / 2 + 1 : 0;
      const int32_t *ks = kstart.data() + (size_t)mi * ni;
      DevMatrix M{};
      M.m = m;
      M.odd = odd;
      M.nk = nk;
      M.ncols = ni;
      M.nlevels = 0;
      M.dblock_begin = (int32_t)P.dblocks.size();
      M.level_begin = (int32_t)P.levels.size();
      M.root_rows = ni;
      M.xrow = -1;
      DevDBlock D{};
      D.row_start = 0;
      D.nrows = nk;
      D.ncols = ni;
      D.out_row = 0;
      D.strip_begin = (int32_t)P.strips.size();
      D.aux = -1;
      const int32_t dblock = (int32_t)P.dblocks.size();
      std::vector<int32_t> rm(2 * (size_t)ni);
      int64_t nnz = 0;
      double cost = 0.0;
      if (nk <= 4) {
        // the whole block dense, nk x ni column-major
        const int64_t data = zeros((size_t)nk * ni);
        P.strips.push_back(DevStrip{0, 0, ni, 0, dblock, 0, data});
        for (int c = 0; c < ni; ++c) {
          const int32_t k0 = std::min(ks[c], nk);
          fill[(size_t)mi * ni + c] = DevDenseFill{data + (int64_t)c * nk + k0, 1, nk - k0};
          rm[2 * c] = D.strip_begin;
          rm[2 * c + 1] = c;
          nnz += nk - k0;
        }
        P.dense_elems += (int64_t)nk * ni;
        cost += (double)nk * ni;
      } else {
        std::vector<double> aux(3 * (size_t)(nk - 2));
        for (int32_t k = 2; k < nk; ++k)
          rec_abg(m, m + odd, k, &aux[3 * (k - 2)], &aux[3 * (k - 2) + 1], &aux[3 * (k - 2) + 2]);
        D.aux = (int64_t)append_f64(P.f64, (const char *)aux.data(), aux.size());
        P.aux_values += (int64_t)aux.size();
        // one strip per run of columns with the same first row
        for (int c0 = 0; c0 < ni;) {
          int c1 = c0 + 1;
          while (c1 < ni && ks[c1] == ks[c0]) ++c1;
          const int32_t rs = std::min(ks[c0], nk), nks = nk - rs, nx = c1 - c0;
          DevStrip S{rs, c0, c1, 0, dblock, 0, 0};
          if (nks > 4) {
            S.kind = 1;
            S.data = zeros(3 * (size_t)nx);
            for (int c = c0; c < c1; ++c) {
              P.f64[S.data + (c - c0)] = z[c] * z[c];
              fill[(size_t)mi * ni + c] = DevDenseFill{S.data + nx + (c - c0), nx, 2};
            }
            P.rec_elems += (int64_t)nks * nx;
            P.rec_columns += nx;
            cost += 2.5 * nks * nx;
          } else if (nks > 0) {
            S.data = zeros((size_t)nks * nx);
            for (int c = c0; c < c1; ++c)
              fill[(size_t)mi * ni + c] = DevDenseFill{S.data + (int64_t)(c - c0) * nks, 1, nks};
            P.dense_elems += (int64_t)nks * nx;
            cost += (double)nks * nx;
          }
          for (int c = c0; c < c1; ++c) {
            rm[2 * c] = (int32_t)P.strips.size();
            rm[2 * c + 1] = c - c0;
          }
          nnz += (int64_t)nks * nx;
          P.strips.push_back(S);
          c0 = c1;
        }
      }
      D.strip_end = (int32_t)P.strips.size();
      P.dblocks.push_back(D);
      M.dblock_end = (int32_t)P.dblocks.size();
      M.root_map = (int64_t)append_i32(P.i32, rm);
      M.cost = cost;
      P.element_count[mi] = nnz;
      P.mats.push_back(M);
    }
  }
  P.max_rows = 0;
  return true;
}

bool compile_resource(const char *data, size_t len, int nside_expect, int lmax_expect,
                      int mmax_expect, HostProgram &P, std::string &err) {
  Reader R{data, len, &err};
  int64_t lmax = R.get<int64_t>(0, "file header");
  int64_t mmax = R.get<int64_t>(8, "file header");
  int64_t nside = R.get<int64_t>(16, "file header");
  if (!R.ok) return false;
  char buf[256];
  if (nside_expect >= 0 && nside != nside_expect) {
    snprintf(buf, sizeof buf, "Incompatible Nside: file has %lld, plan wants %d", (long long)nside,
             nside_expect);
    err = buf;
    return false;
  }
  if (lmax != lmax_expect || mmax != mmax_expect) {
    snprintf(buf, sizeof buf, "Incompatible lmax/mmax: file has %lld/%lld, plan wants %d/%d",
             (long long)lmax, (long long)mmax, lmax_expect, mmax_expect);
    err = buf;
    return false;
  }
  if (nside <= 0 || nside > (1 << 15) || lmax < 0 || mmax > lmax) {
    err = "invalid file header";
    return false;
  }
  P.nside = (int)nside;
  P.lmax = (int)lmax;
  P.mmax = (int)mmax;
  P.element_count.assign(2 * (mmax + 1), 0);
  const int ncols = 2 * (int)nside;
  for (int m = 0; m <= mmax; ++m) {
    for (int odd = 0; odd < 2; ++odd) {
      int64_t start = R.get<int64_t>(24 + 8 * (4 * m + 2 * odd), "offset table");
      int64_t mlen = R.get<int64_t>(24 + 8 * (4 * m + 2 * odd + 1), "offset table");
      if (!R.ok) return false;
      int nk = std::max(0, ((int)lmax - m - odd) / 2 + 1);
      if (lmax - m - odd < 0) nk = 0;
      if (start == 0) {
        snprintf(buf, sizeof buf, "matrix m=%d odd=%d missing from resource file", m, odd);
        err = buf;
        return false;
      }
      if (start < 0 || mlen < 0 || (size_t)start > len || (size_t)mlen > len - (size_t)start) {
        snprintf(buf, sizeof buf, "matrix m=%d odd=%d lies outside the resource file", m, odd);
        err = buf;
        return false;
      }
      Reader Rm{data, (size_t)start + (size_t)mlen, &err};
      if (!compile_matrix(Rm, (size_t)start, m, odd, nk, ncols, P)) return false;
    }
  }
  P.max_rows = 0;
  for (auto &M : P.mats) P.max_rows = std::max(P.max_rows, M.max_rows);
  return true;
}

}  // namespace wm

namespace wm {

// Row groups, column tables, work units and seed bookkeeping of the
// tensor-core path (plan.h).  Matrices of depth 0 (one residual block over
// all rows) and depth 1 (every root a (T, B) pair over two leaves, T blocks
// on rows [0, nk/2), B blocks on [nk/2, nk) -- butterfly.pyx:570-573) are
// taken; anything else stays with the generic kernels.
// Streamed split GEMM tables, tile for tile in the order of the split tile
// lists: residual tiles take consecutive chunks of one A pool (alm2map
// tiles, then map2alm tiles), level tiles point into the sliced W.  The row
// maps give each tile row's destination: alm2map residual rows of q (depth
// 0) or of the X buffer (depth 1), map2alm residual rows of the alm, level
// rows of q (alm2map) or of the X buffer (map2alm).
static void build_stream_tables(HostProgram &P) {
  for (int k = 0; k < 4; ++k) {
    P.stream_tiles[k].clear();
    P.stream_rows[k].clear();
    P.stream_sidx[k].clear();
  }
  auto add = [&](int k, const DevStreamTile &t, const std::vector<int32_t> &rows, const std::vector<int32_t> &sidx) {
    P.stream_tiles[k].push_back(t);
    P.stream_rows[k].insert(P.stream_rows[k].end(), rows.begin(), rows.end());
    P.stream_sidx[k].insert(P.stream_sidx[k].end(), sidx.begin(), sidx.end());
  };
  std::vector<int32_t> rows(kSplitM), sidx(kSplitM);
  int64_t a = 0;
  for (const DevSplitTileA &T : P.stiles_a) {
    const DevGroup &G = P.groups[T.group];
    const DevSplitGroup &S = P.sgroups[T.group];
    const DevMatrix &M = P.mats[G.matrix];
    for (int r = 0; r < kSplitM; ++r) {
      const bool act = r < T.ncols;
      const int32_t gr = act ? P.gcols[G.cols + T.col0 + r].row : 0;
      rows[r] = act ? (int32_t)(G.in_q ? q_row(P, M.m, M.odd, gr) : M.xrow + gr) : -1;
      sidx[r] = act ? (int32_t)(G.cols + T.col0 + r) : -1;
    }
    const int32_t nk = S.nrchunks - T.kc0;
    add(kStreamResA2M, DevStreamTile{a, S.apl + T.kc0, nk, T.group, G.in_q ? 0 : 1, 0}, rows, sidx);
    a += nk;
  }
  for (const DevSplitTileB &T : P.stiles_b) {
    const DevGroup &G = P.groups[T.group];
    const DevSplitGroup &S = P.sgroups[T.group];
    const DevMatrix &M = P.mats[G.matrix];
    const int64_t arow0 = (int64_t)M.m * (2 * P.lmax - M.m + 3) / 2 + M.odd;
    for (int r = 0; r < kSplitM; ++r) {
      const bool act = r < T.nrows;
      rows[r] = act ? (int32_t)(arow0 + 2 * (int64_t)(G.rs + T.row0 + r)) : -1;
      sidx[r] = act ? (int32_t)(S.rowoff + T.row0 + r) : -1;
    }
    add(kStreamResM2A, DevStreamTile{a, S.xpl, S.ncchunks, T.group, 2, 0}, rows, sidx);
    a += S.ncchunks;
  }
  P.stream_res_achunks = a;
  const int32_t ng = (int32_t)P.groups.size();
  for (int dir = 0; dir < 2; ++dir) {
    const bool a2m = dir == 0;
    for (const DevSplitLevelTile &T : a2m ? P.stiles_la : P.stiles_lm) {
      const DevRootUnit &U = P.roots[T.unit];
      const DevPair &pr = P.pairs[U.pair];
      const DevMatrix &M = P.mats[U.matrix];
      const DevSplitRoot &R = P.sroots[T.unit];
      const int32_t nk = a2m ? R.nsc : R.nzc;
      for (int r = 0; r < kSplitM; ++r) {
        const bool act = r < T.nrows;
        const int32_t rr = T.row0 + r;
        int64_t dst = -1;
        if (act && a2m) dst = q_row(P, M.m, M.odd, pr.out_left + rr);
        if (act && !a2m) dst = (int64_t)M.xrow + (rr < pr.kT ? pr.inT + rr : pr.inB + (rr - pr.kT));
        rows[r] = (int32_t)dst;
        sidx[r] = act ? (int32_t)((a2m ? R.rs_a2m : R.rs_m2a) + rr) : -1;
      }
      const int64_t a0 = (a2m ? R.a_a2m : R.a_m2a) + (int64_t)(T.row0 / kSplitM) * nk;
      add(a2m ? kStreamLevelA2M : kStreamLevelM2A,
          DevStreamTile{a0, a2m ? R.b_a2m : R.b_m2a, nk, ng + T.unit, a2m ? 0 : 1, 0}, rows, sidx);
    }
  }
}

// Split-precision residual tables: operand chunk offsets per group and the
// M tiles of both directions, largest K extent first.
static void build_split_tables(HostProgram &P) {
  P.sgroups.clear();
  P.stiles_a.clear();
  P.stiles_b.clear();
  int64_t apl = 0, xpl = 0, rows = 0;
  std::vector<std::pair<int32_t, DevSplitTileA>> ta;
  std::vector<std::pair<int32_t, DevSplitTileB>> tb;
  for (auto &z : P.split_zero) z.clear();
  auto zero = [&](int launch, int64_t buf, int64_t row) {
    P.split_zero[launch].push_back((buf << kZeroBufShift) | row);
  };
  for (int32_t gi = 0; gi < (int32_t)P.groups.size(); ++gi) {
    const DevGroup &G = P.groups[gi];
    DevSplitGroup S{};
    S.nrchunks = (G.nrows + kSplitK - 1) / kSplitK;
    S.ncchunks = (G.ncols + kSplitK - 1) / kSplitK;
    S.apl = apl;
    S.xpl = xpl;
    S.rowoff = rows;
    apl += S.nrchunks;
    xpl += S.ncchunks;
    rows += G.nrows;
    P.sgroups.push_back(S);
    for (int32_t c0 = 0; c0 < G.ncols; c0 += kSplitM) {
      DevSplitTileA T{gi, c0, std::min(kSplitM, G.ncols - c0), G.nrows};
      for (int32_t c = c0; c < c0 + T.ncols; ++c)
        T.kc0 = std::min(T.kc0, P.gcols[G.cols + c].start);
      T.kc0 /= kSplitK;
      if (T.kc0 < S.nrchunks) {
        ta.push_back({S.nrchunks - T.kc0, T});
      } else {
        // no active row in any column of the tile: its outputs are zero
        const DevMatrix &M = P.mats[G.matrix];
        for (int32_t c = c0; c < c0 + T.ncols; ++c) {
          const int32_t gr = P.gcols[G.cols + c].row;
          zero(kStreamResA2M, G.in_q ? 0 : 1, G.in_q ? q_row(P, M.m, M.odd, gr) : M.xrow + gr);
        }
      }
    }
    if (S.ncchunks > 0) {
      for (int32_t r0 = 0; r0 < G.nrows; r0 += kSplitM)
        tb.push_back({S.ncchunks, DevSplitTileB{gi, r0, std::min(kSplitM, G.nrows - r0), 0}});
    } else {
      // no skeleton column: the group's alm rows are zero
      const DevMatrix &M = P.mats[G.matrix];
      const int64_t arow0 = (int64_t)M.m * (2 * P.lmax - M.m + 3) / 2 + M.odd;
      for (int32_t r = 0; r < G.nrows; ++r) zero(kStreamResM2A, 2, arow0 + 2 * (int64_t)(G.rs + r));
    }
  }
  std::stable_sort(ta.begin(), ta.end(), [](const auto &a, const auto &b) { return a.first > b.first; });
  std::stable_sort(tb.begin(), tb.end(), [](const auto &a, const auto &b) { return a.first > b.first; });
  for (auto &t : ta) P.stiles_a.push_back(t.second);
  for (auto &t : tb) P.stiles_b.push_back(t.second);
  P.split_chunks = std::max(apl, xpl);
  P.split_rows = rows;
  // level products of the depth-1 roots
  P.sroots.clear();
  P.stiles_la.clear();
  P.stiles_lm.clear();
  int64_t achunks = 0, lrows = 0, bla = 0, blm = 0;
  std::vector<std::pair<int32_t, DevSplitLevelTile>> la, lm;
  for (int32_t u = 0; u < (int32_t)P.roots.size(); ++u) {
    const DevPair &pr = P.pairs[P.roots[u].pair];
    const int32_t K = pr.kT + pr.kB;
    DevSplitRoot R{};
    R.nzc = (pr.n + kSplitK - 1) / kSplitK;
    R.nsc = (K + kSplitK - 1) / kSplitK;
    const int32_t nzt = (pr.n + kSplitM - 1) / kSplitM, nst = (K + kSplitM - 1) / kSplitM;
    R.a_a2m = achunks;
    achunks += (int64_t)nzt * R.nsc;
    R.a_m2a = achunks;
    achunks += (int64_t)nst * R.nzc;
    R.b_a2m = bla;
    bla += R.nsc;
    R.b_m2a = blm;
    blm += R.nzc;
    R.rs_a2m = lrows;
    lrows += pr.n;
    R.rs_m2a = lrows;
    lrows += K;
    P.sroots.push_back(R);
    if (R.nsc > 0) {
      for (int32_t z0 = 0; z0 < pr.n; z0 += kSplitM)
        la.push_back({R.nsc, DevSplitLevelTile{u, z0, std::min(kSplitM, pr.n - z0), 0}});
    } else {
      // a root without skeleton rows: its q rows are zero
      const DevMatrix &M = P.mats[P.roots[u].matrix];
      for (int32_t z = 0; z < pr.n; ++z) zero(kStreamLevelA2M, 0, q_row(P, M.m, M.odd, pr.out_left + z));
    }
    if (R.nzc > 0)
      for (int32_t s0 = 0; s0 < K; s0 += kSplitM)
        lm.push_back({R.nzc, DevSplitLevelTile{u, s0, std::min(kSplitM, K - s0), 0}});
  }
  std::stable_sort(la.begin(), la.end(), [](const auto &a, const auto &b) { return a.first > b.first; });
  std::stable_sort(lm.begin(), lm.end(), [](const auto &a, const auto &b) { return a.first > b.first; });
  for (auto &t : la) P.stiles_la.push_back(t.second);
  for (auto &t : lm) P.stiles_lm.push_back(t.second);
  P.split_level_achunks = achunks;
  P.split_level_rows = lrows;
  P.split_chunks = std::max(P.split_chunks, std::max(bla, blm));
  build_stream_tables(P);
}

bool build_fast_path(HostProgram &P, std::string &err) {
  P.groups.clear();
  P.gcols.clear();
  P.tiles_a.clear();
  P.tiles_b.clear();
  P.roots.clear();
  P.slow_mats.clear();
  P.nseeds = 0;
  P.xrows = 0;
  P.max_root_k = 0;
  P.max_root_n = 0;
  for (size_t mi = 0; mi < P.mats.size(); ++mi) {
    DevMatrix &M = P.mats[mi];
    M.fast = 0;
    M.xrow = -1;
    if (P.shard_m1 >= 0 && (M.m < P.shard_m0 || M.m >= P.shard_m1)) continue;  // another shard's
    const int nblk = M.dblock_end - M.dblock_begin;
    bool ok = M.nk > 0 && (M.nlevels == 0 || M.nlevels == 1);
    if (ok && M.nlevels == 0) ok = (nblk == 1);
    if (ok && M.nlevels == 1) {
      ok = (nblk % 2 == 0);
      const DevLevel &L = P.levels[M.level_begin];
      ok = ok && (L.pair_end - L.pair_begin) * 2 == nblk;
    }
    // row ranges of the groups
    std::vector<std::pair<int32_t, int32_t>> ranges;
    if (ok) {
      if (M.nlevels == 0) ranges = {{0, M.nk}};
      else ranges = {{0, M.nk / 2}, {M.nk / 2, M.nk}};
      for (int b = 0; b < nblk && ok; ++b) {
        const DevDBlock &D = P.dblocks[M.dblock_begin + b];
        const auto &rg = ranges[M.nlevels == 0 ? 0 : (b % 2)];
        if (D.nrows == 0) continue;
        ok = D.row_start >= rg.first && D.row_start + D.nrows == rg.second;
      }
    }
    if (!ok) {
      P.slow_mats.push_back((int32_t)mi);
      continue;
    }
    M.fast = 1;
    if (M.nlevels == 1) {
      M.xrow = P.xrows;
      P.xrows += M.root_rows;
      const DevLevel &L = P.levels[M.level_begin];
      for (int32_t pi = L.pair_begin; pi < L.pair_end; ++pi) {
        const DevPair &pr = P.pairs[pi];
        if (pr.out_right != pr.out_left + pr.n_left) {
          err = "depth-1 root whose leaves are not adjacent";
          return false;
        }
        P.roots.push_back(DevRootUnit{(int32_t)mi, pi});
        P.max_root_k = std::max(P.max_root_k, pr.kT + pr.kB);
        P.max_root_n = std::max(P.max_root_n, pr.n);
      }
    }
    for (size_t g = 0; g < ranges.size(); ++g) {
      DevGroup G{};
      G.matrix = (int32_t)mi;
      G.rs = ranges[g].first;
      G.nrows = ranges[g].second - ranges[g].first;
      G.cols = (int64_t)P.gcols.size();
      G.in_q = M.nlevels == 0 ? 1 : 0;
      for (int b = 0; b < nblk; ++b) {
        if (M.nlevels == 1 && (size_t)(b % 2) != g) continue;
        const DevDBlock &D = P.dblocks[M.dblock_begin + b];
        const int32_t boff = D.nrows ? D.row_start - G.rs : G.nrows;
        for (int32_t c = 0; c < D.ncols; ++c) {
          DevGCol C{};
          C.row = D.out_row + c;
          C.boff = boff;
          C.aux = D.aux;
          C.start = G.nrows;  // inactive unless a strip covers it
          for (int32_t s = D.strip_begin; s < D.strip_end; ++s) {
            const DevStrip &S = P.strips[s];
            if (c < S.cstart || c >= S.cstop) continue;
            const int32_t nks = D.nrows - S.rstart;
            if (D.nrows == 0 || nks <= 0) break;
            C.start = boff + S.rstart;
            C.kind = S.kind;
            if (S.kind == 0) {
              C.data = S.data + (int64_t)(c - S.cstart) * nks;
            } else {
              C.nx = S.cstop - S.cstart;
              C.data = S.data + (c - S.cstart);
            }
            break;
          }
          P.gcols.push_back(C);
        }
      }
      G.ncols = (int32_t)(P.gcols.size() - G.cols);
      // columns by first active row, so that the column tiles of the
      // tensor-core kernels span similar row ranges
      std::stable_sort(P.gcols.begin() + G.cols, P.gcols.end(),
                       [](const DevGCol &a, const DevGCol &b) { return a.start < b.start; });
      G.nchunks = (G.nrows + kSeedRows - 1) / kSeedRows;
      G.seeds = P.nseeds;
      P.nseeds += 2LL * G.ncols * G.nchunks;
      const int32_t gi = (int32_t)P.groups.size();
      P.groups.push_back(G);
      const int32_t ntiles = (G.ncols + 255) / 256;
      const int32_t width = ntiles ? ((G.ncols + ntiles - 1) / ntiles + 7) & ~7 : 8;
      for (int32_t c0 = 0; c0 < G.ncols; c0 += width) {
        DevTileA T{gi, c0, std::min(width, G.ncols - c0), G.nrows};
        for (int32_t c = c0; c < c0 + T.ncols; ++c)
          T.kstart = std::min(T.kstart, P.gcols[G.cols + c].start);
        T.kstart &= ~3;
        P.tiles_a.push_back(T);
      }
      for (int32_t r0 = 0; r0 < G.nrows; r0 += kPushRows)
        P.tiles_b.push_back(DevTileB{gi, r0, std::min(kPushRows, G.nrows - r0), r0 / kSeedRows});
    }
  }
  build_split_tables(P);
  return true;
}

}  // namespace wm
