// C ABI of libwavemoth_b200.so: the plan object and every extern "C" entry
// point declared in include/wavemoth.h and include/wavemoth_b200.h.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <numeric>
#include <string>
#include <vector>

#include "kernels.h"
#include "plan.h"
#include "program.h"
#include "wavemoth.h"
#include "wavemoth_b200.h"

namespace {

thread_local std::string g_last_error;
std::string g_resource_dir;
int64_t g_device_cap = 0;

int set_error(int code, const std::string &msg) {
  g_last_error = msg;
  return code;
}

struct DeviceArena {
  std::vector<void *> ptrs;
  int64_t bytes = 0;
  ~DeviceArena() {
    for (void *p : ptrs) cudaFree(p);
  }
  template <class T>
  int alloc(T **out, size_t count, const char *what) {
    size_t nbytes = std::max<size_t>(count, 1) * sizeof(T);
    if (g_device_cap > 0 && bytes + (int64_t)nbytes > g_device_cap)
      return set_error(WAVEMOTH_ERR_NOMEM, std::string("device memory cap exceeded allocating ") + what);
    void *p = nullptr;
    cudaError_t e = cudaMalloc(&p, nbytes);
    if (e != cudaSuccess)
      return set_error(WAVEMOTH_ERR_NOMEM, std::string("cudaMalloc(") + what + "): " +
                                               cudaGetErrorString(e));
    ptrs.push_back(p);
    bytes += (int64_t)nbytes;
    *out = (T *)p;
    return 0;
  }
};

}  // namespace

struct _wavemoth_plan {
  int nside = 0, lmax = 0, mmax = 0, nmaps = 0, nvecs = 0, ni = 0;
  int64_t npix = 0, nalm = 0;
  unsigned flags = 0;
  bool analysis = false;          // map2alm plan
  double *host_in = nullptr, *host_out = nullptr;
  int status = 0;
  int phase_shifts = 1;
  int sm_count = 0;
  int grid = 0;

  wm::HostProgram prog;
  DeviceArena arena;
  int64_t program_bytes = 0;
  wm::DevMatrix *d_mats = nullptr;
  wm::DevDBlock *d_dblocks = nullptr;
  wm::DevStrip *d_strips = nullptr;
  wm::DevLevel *d_levels = nullptr;
  wm::DevPair *d_pairs = nullptr;
  double *d_f64 = nullptr;
  int32_t *d_i32 = nullptr;
  int32_t *d_order = nullptr;       // all matrices, largest first (generic kernel over everything)
  int32_t *d_order_slow = nullptr;  // matrices left to the generic kernel by the tensor-core path
  int32_t nslow = 0;
  int32_t *d_counter = nullptr;
  // tensor-core path
  wm::DevGroup *d_groups = nullptr;
  wm::DevGCol *d_gcols = nullptr;
  wm::DevTileA *d_tiles_a = nullptr;
  wm::DevTileB *d_tiles_b = nullptr;
  wm::DevRootUnit *d_roots = nullptr;
  double *d_seeds = nullptr;
  double *d_xbuf = nullptr;
  // split-precision residual path
  bool split = false;
  wm::DevSplitGroup *d_sgroups = nullptr;
  wm::DevSplitTileA *d_stiles_a = nullptr;
  wm::DevSplitTileB *d_stiles_b = nullptr;
  double2 *d_col_scale = nullptr, *d_row_scale = nullptr, *d_vec_scale = nullptr;
  int8_t *d_planes = nullptr;
  wm::DevSplitRoot *d_sroots = nullptr;
  wm::DevSplitLevelTile *d_stiles_la = nullptr, *d_stiles_lm = nullptr;
  int8_t *d_level_a = nullptr;
  double2 *d_level_rs = nullptr;
  int32_t *d_status = nullptr;
  wm::DevRing *d_rings = nullptr;
  wm::DevRingTask *d_ring_tasks = nullptr;
  double *d_twiddles = nullptr, *d_filters = nullptr, *d_ring_aux = nullptr;
  int32_t twlen = 0, max_bluestein = 0;
  int32_t ring_ntasks = 0, ring_smem = 0, nphase_hi = 1;
  double *d_alm = nullptr, *d_map = nullptr, *d_q = nullptr, *d_scratch = nullptr;
  int64_t slot_stride = 0;
  cudaStream_t stream = nullptr;

  // optional per-kernel event timing (wavemoth_plan_timing)
  bool timing = false;
  // kernels launched by executes since the last timing reset
  int64_t kernel_launches = 0;
  struct Span { int kind; cudaEvent_t a, b; };
  std::vector<Span> spans;

  ~_wavemoth_plan() {
    for (auto &s : spans) { cudaEventDestroy(s.a); cudaEventDestroy(s.b); }
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace {

int cuda_check(cudaError_t e, const char *what) {
  if (e == cudaSuccess) return 0;
  return set_error(WAVEMOTH_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

template <class T>
int upload(DeviceArena &A, T **dst, const std::vector<T> &src, const char *what) {
  if (int rc = A.alloc(dst, src.size(), what)) return rc;
  if (!src.empty())
    return cuda_check(cudaMemcpy(*dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice),
                      what);
  return 0;
}

bool read_file(const std::string &path, std::vector<char> &buf, std::string &err) {
  FILE *f = fopen(path.c_str(), "rb");
  if (!f) {
    err = "cannot open resource file " + path;
    return false;
  }
  fseek(f, 0, SEEK_END);
  long n = ftell(f);
  fseek(f, 0, SEEK_SET);
  if (n < 0) {
    fclose(f);
    err = "cannot size resource file " + path;
    return false;
  }
  buf.resize((size_t)n);
  size_t got = n ? fread(buf.data(), 1, (size_t)n, f) : 0;
  fclose(f);
  if (got != (size_t)n) {
    err = "short read of resource file " + path;
    return false;
  }
  return true;
}

struct RingTable {
  std::vector<wm::DevRing> rings;
  std::vector<wm::DevRingTask> tasks;  // by decreasing cost
  int64_t filter_cplx = 0;   // complex entries of all Bluestein filter spectra
  int64_t aux_cplx = 0;      // complex entries of all Bluestein chirp/root tables
  int32_t twlen = 4;         // largest power-of-two table length needed
  int32_t max_bluestein = 0;
  int32_t smem = 0;
  int32_t nphase_hi = 1;
  int64_t max_cta_cplx = 0;  // largest transform buffer of one CTA
};

// Ring geometry (src/wavemoth.c:1199-1232) and the CTA work list of the ring
// kernels: per ring pair, groups of G maps with both hemispheres and
// 2 G x (transform length) within the CTA buffer; transforms longer than half
// the buffer run one map and one hemisphere per CTA.  Ordered by decreasing
// cost so that the long transforms start first.
RingTable ring_table(int nside, int nmaps, int mmax) {
  const int nrings = 4 * nside - 1, mid = 2 * nside - 1;
  std::vector<int64_t> offs(nrings + 1);
  int64_t ipix = 0, npr = 0;
  std::vector<int> num(nrings), den(nrings);
  for (int r = 0; r < nrings; ++r) {
    if (r <= nside - 1) {
      npr += 4;
      num[r] = 1;
      den[r] = 4 * (r + 1);
    } else if (r > 3 * nside - 1) {
      npr -= 4;
      num[r] = 1;
      den[r] = 4 * (nrings - r);
    } else {
      num[r] = r % 2;
      den[r] = 4 * nside;
    }
    offs[r] = ipix;
    ipix += npr;
  }
  offs[nrings] = ipix;
  RingTable T;
  T.rings.resize(2 * nside);
  T.nphase_hi = mmax / 64 + 1;
  int gmax = 1;
  while (gmax < nmaps && gmax < 8) gmax <<= 1;
  struct Item { double cost; wm::DevRingTask t; int64_t cplx; };
  std::vector<Item> items;
  for (int r = 0; r < 2 * nside; ++r) {
    wm::DevRing R{};
    R.n = (int32_t)(offs[mid + r + 1] - offs[mid + r]);
    R.phi_num = num[mid + r];
    R.phi_den = den[mid + r];
    R.off_north = offs[mid - r];
    R.off_south = offs[mid + r];
    const int N = R.n / 2;
    int len = N;
    if (N & (N - 1)) {
      int M = 1;
      while (M < 2 * N - 1) M <<= 1;
      R.bluestein_m = M;
      R.filter = T.filter_cplx;
      T.filter_cplx += M;
      R.aux = T.aux_cplx;
      T.aux_cplx += 2 * N + 1;
      T.max_bluestein = std::max(T.max_bluestein, M);
      len = M;
      T.twlen = std::max(T.twlen, M);
    } else {
      T.twlen = std::max(T.twlen, 2 * N);  // roots e^{2 pi i k / n}, n = 2N
    }
    T.rings[r] = R;
    // both hemispheres in one CTA (lanes = sides x maps) when they fit the
    // buffer; the longest transforms run one hemisphere at a time
    int G = 1, two = 1;
    if (2 * len <= wm::kRingBufferCplx) G = std::min(gmax, wm::kRingBufferCplx / (2 * len));
    else two = 0;
    int lg = 0;
    while ((1 << lg) < G) ++lg;
    const int64_t cplx = (int64_t)G * len << two;
    const double cost = (double)cplx * (R.bluestein_m ? 2.5 : 1.0) + (double)G * (mmax + 1);
    T.max_cta_cplx = std::max(T.max_cta_cplx, cplx);
    for (int g0 = 0; g0 < nmaps; g0 += G)
      items.push_back({cost, wm::DevRingTask{r, g0, lg, two}, cplx});
  }
  std::stable_sort(items.begin(), items.end(), [](const Item &a, const Item &b) { return a.cost > b.cost; });
  int64_t need = 0;
  for (const Item &it : items) {
    T.tasks.push_back(it.t);
    need = std::max(need, it.cplx);
  }
  T.smem = T.tasks.empty() ? 0 : wm::ring_cta_smem(need, T.nphase_hi);
  return T;
}

wm::RingParams ring_params(wavemoth_plan P);

wm::FastParams fast_params(wavemoth_plan P) {
  const auto &G = P->prog;
  wm::FastParams f{};
  f.mats = P->d_mats;
  f.pairs = P->d_pairs;
  f.f64 = P->d_f64;
  f.i32 = P->d_i32;
  f.groups = P->d_groups;
  f.gcols = P->d_gcols;
  f.tiles_a = P->d_tiles_a;
  f.tiles_b = P->d_tiles_b;
  f.roots = P->d_roots;
  f.seeds = P->d_seeds;
  f.ngroups = (int32_t)G.groups.size();
  f.ngcols = (int64_t)G.gcols.size();
  f.ntiles_a = (int32_t)G.tiles_a.size();
  f.ntiles_b = (int32_t)G.tiles_b.size();
  f.nroots = (int32_t)G.roots.size();
  f.max_root_k = G.max_root_k;
  f.max_root_n = G.max_root_n;
  f.lmax = P->lmax;
  f.nvecs = P->nvecs;
  f.ni = P->ni;
  f.xbuf = P->d_xbuf;
  return f;
}

wm::SplitParams split_params(wavemoth_plan P) {
  const auto &G = P->prog;
  wm::SplitParams s{};
  s.mats = P->d_mats;
  s.f64 = P->d_f64;
  s.groups = P->d_groups;
  s.gcols = P->d_gcols;
  s.sgroups = P->d_sgroups;
  s.tiles_a = P->d_stiles_a;
  s.tiles_b = P->d_stiles_b;
  s.ngroups = (int32_t)G.groups.size();
  s.ngcols = (int64_t)G.gcols.size();
  s.ntiles_a = (int32_t)G.stiles_a.size();
  s.ntiles_b = (int32_t)G.stiles_b.size();
  s.seeds = P->d_seeds;
  s.col_scale = P->d_col_scale;
  s.row_scale = P->d_row_scale;
  s.vec_scale = P->d_vec_scale;
  s.planes = P->d_planes;
  s.nrowscale = G.split_rows;
  s.lmax = P->lmax;
  s.nvecs = P->nvecs;
  s.ni = P->ni;
  s.xbuf = P->d_xbuf;
  s.status = P->d_status;
  s.pairs = P->d_pairs;
  s.i32 = P->d_i32;
  s.roots = P->d_roots;
  s.sroots = P->d_sroots;
  s.tiles_la = P->d_stiles_la;
  s.tiles_lm = P->d_stiles_lm;
  s.nroots = (int32_t)G.roots.size();
  s.ntiles_la = (int32_t)G.stiles_la.size();
  s.ntiles_lm = (int32_t)G.stiles_lm.size();
  s.level_a = P->d_level_a;
  s.level_rs = P->d_level_rs;
  return s;
}

wavemoth_plan make_plan(bool analysis, int Nside, int lmax, int mmax, int nmaps, double *input,
                        double *output, int ordering, unsigned flags, const char *resource_filename) {
  if (nmaps <= 0 || lmax < 0 || mmax != lmax || ordering != WAVEMOTH_MMAJOR) {
    set_error(WAVEMOTH_ERR_ARG, "invalid plan arguments (need nmaps > 0, mmax == lmax >= 0, "
                                "ordering WAVEMOTH_MMAJOR)");
    return nullptr;
  }
  std::string path;
  if (resource_filename) {
    path = resource_filename;
  } else {
    if (Nside <= 0 || g_resource_dir.empty()) {
      set_error(WAVEMOTH_ERR_ARG, "no resource file given and wavemoth_configure not called");
      return nullptr;
    }
    path = g_resource_dir + "/rev1/" + std::to_string(Nside) + ".dat";
  }
  std::vector<char> file;
  std::string err;
  if (!read_file(path, file, err)) {
    set_error(WAVEMOTH_ERR_RESOURCE, err);
    return nullptr;
  }
  auto *P = new _wavemoth_plan();
  if (!wm::compile_resource(file.data(), file.size(), Nside, lmax, mmax, P->prog, err)) {
    set_error(WAVEMOTH_ERR_RESOURCE, path + ": " + err);
    delete P;
    return nullptr;
  }
  file.clear();
  file.shrink_to_fit();
  P->nside = P->prog.nside;
  P->lmax = lmax;
  P->mmax = mmax;
  P->nmaps = nmaps;
  P->nvecs = 2 * nmaps;
  P->ni = 2 * P->nside;
  P->npix = 12LL * P->nside * P->nside;
  P->nalm = (int64_t)(lmax + 1) * (lmax + 2) / 2;
  P->flags = flags;
  P->analysis = analysis;
  P->host_in = input;
  P->host_out = output;

  int dev = 0;
  if (cuda_check(cudaGetDevice(&dev), "cudaGetDevice") ||
      cuda_check(cudaDeviceGetAttribute(&P->sm_count, cudaDevAttrMultiProcessorCount, dev),
                 "cudaDeviceGetAttribute")) {
    delete P;
    return nullptr;
  }
  auto &G = P->prog;
  if (!wm::build_fast_path(G, err)) {
    set_error(WAVEMOTH_ERR_RESOURCE, path + ": " + err);
    delete P;
    return nullptr;
  }
  // processing order: largest matrices first
  std::vector<int32_t> order(G.mats.size());
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(),
                   [&](int a, int b) { return G.mats[a].cost > G.mats[b].cost; });
  const int nmats = (int)G.mats.size();
  P->grid = std::max(1, std::min(nmats, 2 * P->sm_count));
  P->slot_stride = 2 * (int64_t)std::max<int32_t>(G.max_rows, 1) * P->nvecs;
  int rc = 0;
  DeviceArena &A = P->arena;
  rc = rc ? rc : upload(A, &P->d_mats, G.mats, "matrices");
  rc = rc ? rc : upload(A, &P->d_dblocks, G.dblocks, "residual blocks");
  rc = rc ? rc : upload(A, &P->d_strips, G.strips, "strips");
  rc = rc ? rc : upload(A, &P->d_levels, G.levels, "levels");
  rc = rc ? rc : upload(A, &P->d_pairs, G.pairs, "pairs");
  rc = rc ? rc : upload(A, &P->d_f64, G.f64, "f64 arena");
  rc = rc ? rc : upload(A, &P->d_i32, G.i32, "i32 arena");
  rc = rc ? rc : upload(A, &P->d_order, order, "order");
  {
    std::vector<int32_t> slow;
    std::vector<char> is_slow(G.mats.size(), 0);
    for (int32_t mi : G.slow_mats) is_slow[mi] = 1;
    for (int32_t mi : order)
      if (is_slow[mi]) slow.push_back(mi);
    P->nslow = (int32_t)slow.size();
    rc = rc ? rc : upload(A, &P->d_order_slow, slow, "slow order");
  }
  rc = rc ? rc : upload(A, &P->d_groups, G.groups, "groups");
  rc = rc ? rc : upload(A, &P->d_gcols, G.gcols, "group columns");
  rc = rc ? rc : upload(A, &P->d_tiles_a, G.tiles_a, "alm2map tiles");
  rc = rc ? rc : upload(A, &P->d_tiles_b, G.tiles_b, "map2alm tiles");
  rc = rc ? rc : upload(A, &P->d_roots, G.roots, "roots");
  rc = rc ? rc : A.alloc(&P->d_seeds, (size_t)std::max<int64_t>(G.nseeds, 1), "recurrence seeds");
  P->program_bytes = A.bytes;
  rc = rc ? rc : A.alloc(&P->d_xbuf, (size_t)std::max<int64_t>(G.xrows, 1) * P->nvecs, "X buffer");
  {
    RingTable RT = ring_table(P->nside, nmaps, mmax);
    if (!rc && RT.max_cta_cplx > wm::kRingBufferCplx)
      rc = set_error(WAVEMOTH_ERR_ARG, "ring transforms longer than 8192 points (nside > 2048) are not supported");
    P->twlen = RT.twlen;
    P->max_bluestein = RT.max_bluestein;
    P->ring_ntasks = (int32_t)RT.tasks.size();
    P->ring_smem = RT.smem;
    P->nphase_hi = RT.nphase_hi;
    rc = rc ? rc : upload(A, &P->d_rings, RT.rings, "ring table");
    rc = rc ? rc : upload(A, &P->d_ring_tasks, RT.tasks, "ring work list");
    rc = rc ? rc : A.alloc(&P->d_twiddles, (size_t)RT.twlen, "twiddle table");
    rc = rc ? rc : A.alloc(&P->d_filters, (size_t)std::max<int64_t>(2 * RT.filter_cplx, 2),
                           "Bluestein filters");
    rc = rc ? rc : A.alloc(&P->d_ring_aux, (size_t)std::max<int64_t>(2 * RT.aux_cplx, 2),
                           "Bluestein chirps");
  }
  P->split = (flags & WAVEMOTH_PRECISION_SPLIT) != 0;
  if (P->split) {
    rc = rc ? rc : upload(A, &P->d_sgroups, G.sgroups, "split groups");
    rc = rc ? rc : upload(A, &P->d_stiles_a, G.stiles_a, "split alm2map tiles");
    rc = rc ? rc : upload(A, &P->d_stiles_b, G.stiles_b, "split map2alm tiles");
    rc = rc ? rc : A.alloc(&P->d_col_scale, (size_t)std::max<int64_t>((int64_t)G.gcols.size(), 1), "column scales");
    rc = rc ? rc : A.alloc(&P->d_row_scale, (size_t)std::max<int64_t>(G.split_rows, 1), "row scales");
    rc = rc ? rc : A.alloc(&P->d_vec_scale, (size_t)std::max<size_t>(G.groups.size() + G.roots.size(), 1) *
                                                wm::kSplitN, "vector scales");
    rc = rc ? rc : upload(A, &P->d_sroots, G.sroots, "split roots");
    rc = rc ? rc : upload(A, &P->d_stiles_la, G.stiles_la, "split alm2map level tiles");
    rc = rc ? rc : upload(A, &P->d_stiles_lm, G.stiles_lm, "split map2alm level tiles");
    rc = rc ? rc : A.alloc(&P->d_level_a,
                           (size_t)std::max<int64_t>(G.split_level_achunks, 1) * wm::kSplitSlices * wm::kSplitM *
                               wm::kSplitK, "sliced interpolation matrices");
    rc = rc ? rc : A.alloc(&P->d_level_rs, (size_t)std::max<int64_t>(G.split_level_rows, 1),
                           "interpolation row scales");
    rc = rc ? rc : A.alloc(&P->d_planes, (size_t)std::max<int64_t>(G.split_chunks, 1) * wm::kSplitPlane,
                           "operand slices");
  }
  rc = rc ? rc : A.alloc(&P->d_status, 1, "status word");
  rc = rc ? rc : A.alloc(&P->d_counter, 1, "counter");
  rc = rc ? rc : A.alloc(&P->d_q, (size_t)2 * (mmax + 1) * P->ni * P->nvecs, "q buffer");
  rc = rc ? rc : A.alloc(&P->d_scratch, (size_t)P->grid * P->slot_stride, "butterfly scratch");
  if (!(flags & WAVEMOTH_DEVICE_POINTERS)) {
    rc = rc ? rc : A.alloc(&P->d_alm, (size_t)P->nalm * P->nvecs, "alm buffer");
    rc = rc ? rc : A.alloc(&P->d_map, (size_t)P->npix * nmaps, "map buffer");
  }
  rc = rc ? rc : cuda_check(cudaStreamCreateWithFlags(&P->stream, cudaStreamNonBlocking),
                            "cudaStreamCreate");
  if (!rc) {
    wm::RingParams rp = ring_params(P);
    rc = cuda_check(wm::launch_ring_setup(rp, P->d_twiddles, P->max_bluestein ? P->d_filters : nullptr,
                                          P->d_ring_aux, P->stream), "ring setup launch");
    if (!rc) rc = cuda_check(cudaStreamSynchronize(P->stream), "ring setup");
  }
  if (!rc && G.nseeds > 0) {
    wm::FastParams fp = fast_params(P);
    fp.seeds_out = P->d_seeds;
    rc = cuda_check(wm::launch_seeds(fp, P->stream), "seed kernel launch");
    if (!rc) rc = cuda_check(cudaStreamSynchronize(P->stream), "seed kernel");
  }
  if (!rc) rc = cuda_check(cudaMemsetAsync(P->d_status, 0, sizeof(int32_t), P->stream), "status reset");
  if (!rc && P->split && !G.gcols.empty()) {
    // per-column and per-row maxima of P (scratch freed after use)
    unsigned long long *colmax = nullptr, *rowmax = nullptr;
    const size_t nc = G.gcols.size(), nr = (size_t)std::max<int64_t>(G.split_rows, 1);
    rc = cuda_check(cudaMalloc(&colmax, nc * sizeof(unsigned long long)), "scale scratch");
    if (!rc) rc = cuda_check(cudaMalloc(&rowmax, nr * sizeof(unsigned long long)), "scale scratch");
    if (!rc) rc = cuda_check(cudaMemsetAsync(rowmax, 0, nr * sizeof(unsigned long long), P->stream), "scale scratch");
    if (!rc) {
      wm::SplitParams sp = split_params(P);
      sp.colmax = colmax;
      sp.rowmax = rowmax;
      rc = cuda_check(wm::launch_split_scales(sp, P->stream), "split scale launch");
      if (!rc) rc = cuda_check(wm::launch_level_slices(sp, P->stream), "level slice launch");
      if (!rc) rc = cuda_check(cudaStreamSynchronize(P->stream), "split scales");
    }
    cudaFree(colmax);
    cudaFree(rowmax);
  }
  if (rc) {
    delete P;
    return nullptr;
  }
  // host-side tables are no longer needed except element counts
  G.dblocks.clear(); G.dblocks.shrink_to_fit();
  G.strips.clear(); G.strips.shrink_to_fit();
  G.pairs.clear(); G.pairs.shrink_to_fit();
  G.f64.clear(); G.f64.shrink_to_fit();
  G.i32.clear(); G.i32.shrink_to_fit();
  G.gcols.clear(); G.gcols.shrink_to_fit();
  G.tiles_a.shrink_to_fit();
  return P;
}

wm::LegendreParams legendre_params(wavemoth_plan P) {
  wm::LegendreParams p{};
  p.mats = P->d_mats;
  p.dblocks = P->d_dblocks;
  p.strips = P->d_strips;
  p.levels = P->d_levels;
  p.pairs = P->d_pairs;
  p.f64 = P->d_f64;
  p.i32 = P->d_i32;
  p.order = P->d_order;
  p.nmats = (int32_t)P->prog.mats.size();
  p.lmax = P->lmax;
  p.nvecs = P->nvecs;
  p.ni = P->ni;
  p.scratch = P->d_scratch;
  p.slot_stride = P->slot_stride;
  p.counter = P->d_counter;
  return p;
}

}  // namespace

namespace wm {

int set_last_error(int code, const std::string &msg) { return set_error(code, msg); }

// Legendre kernel parameters of a plan (program tables, sizes, grid) without
// any buffers bound; used by entry points that bring their own buffers.
bool plan_legendre_params(wavemoth_plan plan, LegendreParams &p, int &grid, std::string &err) {
  if (!plan) {
    err = "NULL plan";
    return false;
  }
  p = legendre_params(plan);
  grid = plan->grid;
  return true;
}

}  // namespace wm

namespace {

wm::RingParams ring_params(wavemoth_plan P) {
  wm::RingParams r{};
  r.rings = P->d_rings;
  r.ni = P->ni;
  r.nside = P->nside;
  r.mmax = P->mmax;
  r.nmaps = P->nmaps;
  r.nvecs = P->nvecs;
  r.scale = 4.0 * 3.14159265358979323846 / (double)P->npix;
  r.phase_shifts = P->phase_shifts;
  r.twiddles = reinterpret_cast<const double2 *>(P->d_twiddles);
  r.twlen = P->twlen;
  r.filters = P->d_filters;
  r.aux = reinterpret_cast<const double2 *>(P->d_ring_aux);
  r.max_bluestein_m = P->max_bluestein;
  r.tasks = P->d_ring_tasks;
  r.ntasks = P->ring_ntasks;
  r.smem = P->ring_smem;
  r.nphase_hi = P->nphase_hi;
  return r;
}

// kinds: 0 Legendre alm2map, 1 Legendre map2alm, 2 ring synthesis, 3 ring analysis
int span_begin(wavemoth_plan P, int kind, cudaStream_t st) {
  if (!P->timing) return -1;
  _wavemoth_plan::Span s{kind, nullptr, nullptr};
  if (cudaEventCreate(&s.a) != cudaSuccess || cudaEventCreate(&s.b) != cudaSuccess) return -1;
  cudaEventRecord(s.a, st);
  P->spans.push_back(s);
  return (int)P->spans.size() - 1;
}

void span_end(wavemoth_plan P, int idx, cudaStream_t st) {
  if (idx >= 0) cudaEventRecord(P->spans[idx].b, st);
}

int fast_grid(wavemoth_plan P, int units) {
  return std::max(1, std::min(units, 4 * P->sm_count));
}

// Split-precision residual products, kSplitN vectors per pass: operand
// slices of the pass, then the tensor-core GEMM of every group tile.
int run_split(wavemoth_plan P, bool alm2map, const double *alm_in, double *alm_out, const double *q_in,
              double *q_out, cudaStream_t st) {
  const auto &G = P->prog;
  if (G.groups.empty()) return 0;
  wm::SplitParams s = split_params(P);
  s.alm_in = alm_in;
  s.alm_out = alm_out;
  s.q_in = q_in;
  s.q = q_out;
  const int nt = alm2map ? s.ntiles_a : s.ntiles_b;
  const int nl = alm2map ? s.ntiles_la : s.ntiles_lm;
  const int gop = std::min((int)G.groups.size(), 8 * P->sm_count);
  const int gop_l = std::min(std::max(s.nroots, 1), 8 * P->sm_count);
  for (int v0 = 0; v0 < P->nvecs; v0 += wm::kSplitN) {
    s.v0 = v0;
    int rc = 0;
    // alm2map: residual (alm -> X, q) then levels (X -> q); map2alm reversed
    auto residual = [&]() {
      rc = cuda_check(wm::launch_split(alm2map ? 0 : 2, s, gop, st), "operand slice launch");
      P->kernel_launches++;
      if (!rc && nt) {
        rc = cuda_check(wm::launch_split(alm2map ? 1 : 3, s, std::min(nt, P->sm_count), st), "split GEMM launch");
        P->kernel_launches++;
      }
    };
    auto levels = [&]() {
      if (!nl) return;
      rc = cuda_check(wm::launch_split(alm2map ? 4 : 6, s, gop_l, st), "level operand slice launch");
      P->kernel_launches++;
      if (!rc) {
        rc = cuda_check(wm::launch_split(alm2map ? 5 : 7, s, std::min(nl, P->sm_count), st), "level GEMM launch");
        P->kernel_launches++;
      }
    };
    if (alm2map) {
      residual();
      if (!rc) levels();
    } else {
      levels();
      if (!rc) residual();
    }
    if (rc) return rc;
  }
  return 0;
}

int run_legendre(wavemoth_plan P, bool alm2map, const double *alm_in, double *alm_out,
                 const double *q_in, double *q_out, cudaStream_t st) {
  const auto &G = P->prog;
  int sp = span_begin(P, alm2map ? 0 : 1, st);
  int rc = 0;
  wm::FastParams f = fast_params(P);
  f.alm_in = alm_in;
  f.alm_out = alm_out;
  f.q_in = q_in;
  f.q = q_out;
  const int nta = (int)G.tiles_a.size(), ntb = (int)G.tiles_b.size(), nr = (int)G.roots.size();
  if (P->split) {
    rc = run_split(P, alm2map, alm_in, alm_out, q_in, q_out, st);
  } else if (alm2map) {
    if (nta) rc = cuda_check(wm::launch_fast(0, f, fast_grid(P, nta), st), "alm2map residual launch");
    if (!rc && nr) rc = cuda_check(wm::launch_fast(1, f, fast_grid(P, nr), st), "alm2map level launch");
    P->kernel_launches += (nta > 0) + (nr > 0);
  } else {
    if (nr) rc = cuda_check(wm::launch_fast(2, f, fast_grid(P, nr), st), "map2alm level launch");
    if (!rc && ntb) rc = cuda_check(wm::launch_fast(3, f, fast_grid(P, ntb), st), "map2alm residual launch");
    P->kernel_launches += (ntb > 0) + (nr > 0);
  }
  if (!rc && P->nslow > 0) {
    wm::LegendreParams p = legendre_params(P);
    p.order = P->d_order_slow;
    p.nmats = P->nslow;
    p.alm_in = alm_in;
    p.alm_out = alm_out;
    p.q_in = q_in;
    p.q_out = q_out;
    rc = cuda_check(cudaMemsetAsync(P->d_counter, 0, sizeof(int32_t), st), "counter reset");
    if (!rc)
      rc = cuda_check(wm::launch_legendre(alm2map, p, std::min(P->grid, std::max(1, (int)P->nslow)), st),
                      "Legendre kernel launch");
    P->kernel_launches++;
  }
  span_end(P, sp, st);
  return rc;
}

int run_alm2map(wavemoth_plan P, const double *alm, double *map, cudaStream_t st) {
  if (int rc = run_legendre(P, true, alm, nullptr, nullptr, P->d_q, st)) return rc;
  wm::RingParams r = ring_params(P);
  r.q = P->d_q;
  r.map = map;
  int sp = span_begin(P, 2, st);
  int rc = cuda_check(wm::launch_ring_synthesis(r, st), "ring synthesis launch");
  P->kernel_launches += r.ntasks > 0;
  span_end(P, sp, st);
  return rc;
}

int run_map2alm(wavemoth_plan P, const double *map, double *alm, cudaStream_t st) {
  wm::RingParams r = ring_params(P);
  r.map_in = map;
  r.q_out = P->d_q;
  int sp = span_begin(P, 3, st);
  int rc0 = cuda_check(wm::launch_ring_analysis(r, st), "ring analysis launch");
  P->kernel_launches += r.ntasks > 0;
  span_end(P, sp, st);
  if (rc0) return rc0;
  return run_legendre(P, false, nullptr, alm, P->d_q, nullptr, st);
}

// Reads (and clears) the device status word; the stream must be idle.
int device_status(wavemoth_plan P) {
  int32_t st = 0;
  int rc = cuda_check(cudaMemcpy(&st, P->d_status, sizeof(st), cudaMemcpyDeviceToHost), "status read");
  if (rc) return rc;
  if (st == 0) return 0;
  cudaMemset(P->d_status, 0, sizeof(st));
  return set_error(WAVEMOTH_ERR_DEVICE, st == wm::kStatusTimeout ? "a kernel's bounded wait expired"
                                                                 : "a kernel reported a bad program table");
}

int finish(wavemoth_plan P, int rc) {
  P->status = rc;
  return rc;
}

int host_execute(wavemoth_plan P) {
  cudaStream_t st = P->stream;
  const bool devptr = (P->flags & WAVEMOTH_DEVICE_POINTERS) != 0;
  const size_t alm_bytes = (size_t)P->nalm * P->nvecs * sizeof(double);
  const size_t map_bytes = (size_t)P->npix * P->nmaps * sizeof(double);
  if (!P->host_in || !P->host_out)
    return set_error(WAVEMOTH_ERR_ARG, "plan has no bound input/output buffers");
  int rc = 0;
  if (!P->analysis) {
    const double *alm = devptr ? P->host_in : P->d_alm;
    double *map = devptr ? P->host_out : P->d_map;
    if (!devptr)
      rc = cuda_check(cudaMemcpyAsync(P->d_alm, P->host_in, alm_bytes, cudaMemcpyHostToDevice, st),
                      "alm upload");
    rc = rc ? rc : run_alm2map(P, alm, map, st);
    if (!devptr && !rc)
      rc = cuda_check(cudaMemcpyAsync(P->host_out, P->d_map, map_bytes, cudaMemcpyDeviceToHost, st),
                      "map download");
  } else {
    const double *map = devptr ? P->host_in : P->d_map;
    double *alm = devptr ? P->host_out : P->d_alm;
    if (!devptr)
      rc = cuda_check(cudaMemcpyAsync(P->d_map, P->host_in, map_bytes, cudaMemcpyHostToDevice, st),
                      "map upload");
    rc = rc ? rc : run_map2alm(P, map, alm, st);
    if (!devptr && !rc)
      rc = cuda_check(cudaMemcpyAsync(P->host_out, P->d_alm, alm_bytes, cudaMemcpyDeviceToHost, st),
                      "alm download");
  }
  if (!rc) rc = cuda_check(cudaStreamSynchronize(st), "execute");
  if (!rc) rc = device_status(P);
  return rc;
}

}  // namespace

extern "C" {

const char *wavemoth_last_error(void) { return g_last_error.c_str(); }

void wavemoth_configure(char *resource_dir) { g_resource_dir = resource_dir ? resource_dir : ""; }

wavemoth_plan wavemoth_plan_to_healpix(int Nside, int lmax, int mmax, int nmaps, int nthreads,
                                       double *input, double *output, int ordering,
                                       unsigned flags, char *resource_filename) {
  (void)nthreads;
  return make_plan(false, Nside, lmax, mmax, nmaps, input, output, ordering, flags,
                   resource_filename);
}

wavemoth_plan wavemoth_plan_from_healpix(int Nside, int lmax, int mmax, int nmaps, int nthreads,
                                         double *input, double *output, int ordering,
                                         unsigned flags, char *resource_filename) {
  (void)nthreads;
  return make_plan(true, Nside, lmax, mmax, nmaps, input, output, ordering, flags,
                   resource_filename);
}

void wavemoth_destroy_plan(wavemoth_plan plan) {
  if (!plan) return;
  if (plan->stream) cudaStreamSynchronize(plan->stream);
  delete plan;
}

void wavemoth_execute(wavemoth_plan plan) {
  if (!plan) {
    set_error(WAVEMOTH_ERR_ARG, "NULL plan");
    return;
  }
  finish(plan, host_execute(plan));
}

int wavemoth_plan_status(wavemoth_plan plan) { return plan ? plan->status : WAVEMOTH_ERR_ARG; }

int wavemoth_plan_device_status(wavemoth_plan plan, void *stream) {
  if (!plan) return set_error(WAVEMOTH_ERR_ARG, "NULL plan");
  if (int rc = cuda_check(cudaStreamSynchronize((cudaStream_t)stream), "device status")) return rc;
  return finish(plan, device_status(plan));
}

int64_t wavemoth_get_legendre_flops(wavemoth_plan plan, int m, int odd) {
  if (!plan || m < 0 || m > plan->mmax || odd < 0 || odd > 1) return -1;
  return plan->prog.element_count[2 * m + odd] * 2 * 2;
}

int wavemoth_query_resourcefile(char *filename, int *out_Nside, int *out_lmax) {
  if (!filename) return -1;
  FILE *f = fopen(filename, "rb");
  if (!f) return -1;
  int64_t fields[3];
  size_t got = fread(fields, sizeof(fields), 1, f);
  fclose(f);
  if (got != 1) {
    set_error(WAVEMOTH_ERR_RESOURCE, std::string("could not read file header: ") + filename);
    return -1;
  }
  *out_lmax = (int)fields[0];
  *out_Nside = (int)fields[2];
  return 0;
}

int wavemoth_execute_alm2map_device(wavemoth_plan plan, const double *alm, double *map,
                                    void *stream) {
  if (!plan || !alm || !map) return set_error(WAVEMOTH_ERR_ARG, "NULL plan or buffer");
  return finish(plan, run_alm2map(plan, alm, map, (cudaStream_t)stream));
}

int wavemoth_execute_map2alm_device(wavemoth_plan plan, const double *map, double *alm,
                                    void *stream) {
  if (!plan || !alm || !map) return set_error(WAVEMOTH_ERR_ARG, "NULL plan or buffer");
  return finish(plan, run_map2alm(plan, map, alm, (cudaStream_t)stream));
}

void wavemoth_perform_legendre_transforms(wavemoth_plan plan) {
  if (!plan) return;
  int rc = 0;
  if (plan->analysis) {
    rc = set_error(WAVEMOTH_ERR_ARG, "perform_legendre_transforms needs an alm2map plan");
  } else if (plan->flags & WAVEMOTH_DEVICE_POINTERS) {
    rc = run_legendre(plan, true, plan->host_in, nullptr, nullptr, plan->d_q, plan->stream);
  } else {
    rc = cuda_check(cudaMemcpyAsync(plan->d_alm, plan->host_in,
                                    (size_t)plan->nalm * plan->nvecs * sizeof(double),
                                    cudaMemcpyHostToDevice, plan->stream),
                    "alm upload");
    rc = rc ? rc : run_legendre(plan, true, plan->d_alm, nullptr, nullptr, plan->d_q, plan->stream);
  }
  if (!rc) rc = cuda_check(cudaStreamSynchronize(plan->stream), "Legendre transforms");
  finish(plan, rc);
}

void wavemoth_perform_backward_ffts(wavemoth_plan plan) {
  if (!plan) return;
  int rc = 0;
  if (plan->analysis) {
    rc = set_error(WAVEMOTH_ERR_ARG, "perform_backward_ffts needs an alm2map plan");
  } else {
    const bool devptr = (plan->flags & WAVEMOTH_DEVICE_POINTERS) != 0;
    wm::RingParams r = ring_params(plan);
    r.q = plan->d_q;
    r.map = devptr ? plan->host_out : plan->d_map;
    rc = cuda_check(wm::launch_ring_synthesis(r, plan->stream), "ring synthesis launch");
    plan->kernel_launches += r.ntasks > 0;
    if (!rc && !devptr)
      rc = cuda_check(cudaMemcpyAsync(plan->host_out, plan->d_map,
                                      (size_t)plan->npix * plan->nmaps * sizeof(double),
                                      cudaMemcpyDeviceToHost, plan->stream),
                      "map download");
    if (!rc) rc = cuda_check(cudaStreamSynchronize(plan->stream), "backward FFTs");
  }
  finish(plan, rc);
}

void wavemoth_disable_phase_shifting(wavemoth_plan plan) {
  if (plan) plan->phase_shifts = 0;
}

int wavemoth_get_work(wavemoth_plan plan, double *out) {
  if (!plan || !out) return set_error(WAVEMOTH_ERR_ARG, "NULL plan or buffer");
  size_t n = (size_t)2 * (plan->mmax + 1) * plan->ni * plan->nvecs;
  int rc = cuda_check(cudaMemcpyAsync(out, plan->d_q, n * sizeof(double), cudaMemcpyDeviceToHost,
                                      plan->stream), "work download");
  if (!rc) rc = cuda_check(cudaStreamSynchronize(plan->stream), "work download");
  return rc;
}

int wavemoth_plan_nmaps(wavemoth_plan plan) { return plan ? plan->nmaps : -1; }
int wavemoth_plan_nside(wavemoth_plan plan) { return plan ? plan->nside : -1; }
int wavemoth_plan_lmax(wavemoth_plan plan) { return plan ? plan->lmax : -1; }
int64_t wavemoth_plan_device_bytes(wavemoth_plan plan) { return plan ? plan->arena.bytes : -1; }
int64_t wavemoth_plan_program_bytes(wavemoth_plan plan) { return plan ? plan->program_bytes : -1; }

void wavemoth_set_device_memory_cap(int64_t bytes) { g_device_cap = bytes; }

int wavemoth_plan_timing(wavemoth_plan plan, int mode, double *out) {
  if (!plan) return set_error(WAVEMOTH_ERR_ARG, "NULL plan");
  if (mode == 0 || mode == 1) {
    if (plan->stream) cudaStreamSynchronize(plan->stream);
    for (auto &s : plan->spans) { cudaEventDestroy(s.a); cudaEventDestroy(s.b); }
    plan->spans.clear();
    plan->timing = (mode == 1);
    plan->kernel_launches = 0;
    return 0;
  }
  if (mode != 2 || !out) return set_error(WAVEMOTH_ERR_ARG, "invalid timing mode");
  for (int i = 0; i < 8; ++i) out[i] = 0.0;
  for (auto &s : plan->spans) {
    if (int rc = cuda_check(cudaEventSynchronize(s.b), "timing event")) return rc;
    float ms = 0.f;
    if (int rc = cuda_check(cudaEventElapsedTime(&ms, s.a, s.b), "timing event")) return rc;
    out[s.kind] += ms;
    out[4 + s.kind] += 1.0;
  }
  return 0;
}

int64_t wavemoth_plan_kernel_launches(wavemoth_plan plan) { return plan ? plan->kernel_launches : -1; }

int wavemoth_plan_work(wavemoth_plan plan, int nmaps, double *out) {
  if (!plan || !out || nmaps <= 0) return set_error(WAVEMOTH_ERR_ARG, "invalid arguments");
  const auto &G = plan->prog;
  const double nvecs = 2.0 * nmaps;
  // Legendre: multiply-adds of the interpolation and residual products, plus
  // 5 flops per recurrence element (shared by all vectors)
  out[0] = 2.0 * nvecs * (double)(G.interp_elems + G.rec_elems + G.dense_elems) + 5.0 * (double)G.rec_elems;
  // compressed-matrix bytes one direction streams: interpolants (one copy),
  // dense residual values, x2/P0/P1 per recurrence column, coefficients
  out[1] = 8.0 * (double)(G.interp_elems + G.dense_elems + 3 * G.rec_columns + G.aux_values);
  // vector traffic of one Legendre launch: alm in (or out) and q out (or in)
  const double nalm = (double)plan->nalm, nq = 2.0 * (plan->mmax + 1) * plan->ni;
  out[2] = 8.0 * nvecs * (nalm + nq);
  // ring kernels: q in (or out) and the maps out (or in)
  out[3] = 8.0 * (nvecs * nq + (double)plan->npix * nmaps);
  out[4] = (double)G.interp_elems;
  out[5] = (double)G.rec_elems;
  out[6] = (double)G.dense_elems;
  out[7] = (double)plan->grid;
  // split path: 64-row (or 64-column) K chunks of 128-row M tiles; per K
  // step of 32, nine MMAs with N summing to 1664 (six slices, i + j <= 6)
  double ea = 0.0, eb = 0.0, la = 0.0, lb = 0.0;
  for (const auto &T : G.stiles_a) ea += (double)(G.sgroups[T.group].nrchunks - T.kc0);
  for (const auto &T : G.stiles_b) eb += (double)G.sgroups[T.group].ncchunks;
  for (const auto &T : G.stiles_la) la += (double)G.sroots[T.unit].nsc;
  for (const auto &T : G.stiles_lm) lb += (double)G.sroots[T.unit].nzc;
  const double chunk = (double)wm::kSplitM * wm::kSplitK;
  const double passes = (double)((2 * nmaps + wm::kSplitN - 1) / wm::kSplitN);
  const double ops_per_elem = 2.0 * 1664.0;  // per element of an A chunk (M x K), all slice windows
  out[8] = ea * chunk;
  out[9] = eb * chunk;
  out[10] = (ea + la) * chunk * ops_per_elem * passes;
  out[11] = (eb + lb) * chunk * ops_per_elem * passes;
  return 0;
}

int wavemoth_check_resourcefile(char *filename, int Nside, int lmax, int64_t *out_stats) {
  if (!filename) return set_error(WAVEMOTH_ERR_ARG, "NULL file name");
  std::vector<char> file;
  std::string err;
  if (!read_file(filename, file, err)) return set_error(WAVEMOTH_ERR_RESOURCE, err);
  wm::HostProgram P;
  if (!wm::compile_resource(file.data(), file.size(), Nside, lmax, lmax, P, err))
    return set_error(WAVEMOTH_ERR_RESOURCE, std::string(filename) + ": " + err);
  if (!wm::build_fast_path(P, err))
    return set_error(WAVEMOTH_ERR_RESOURCE, std::string(filename) + ": " + err);
  if (out_stats) {
    out_stats[0] = (int64_t)P.mats.size();
    out_stats[1] = (int64_t)P.dblocks.size();
    out_stats[2] = (int64_t)P.strips.size();
    out_stats[3] = (int64_t)P.levels.size();
    out_stats[4] = (int64_t)P.pairs.size();
    out_stats[5] = (int64_t)P.f64.size() * 8;
    out_stats[6] = (int64_t)P.i32.size() * 4;
    out_stats[7] = P.max_rows;
  }
  return 0;
}

wavemoth_grid_info *wavemoth_create_healpix_grid_info(int Nside) {
  if (Nside <= 0 || Nside > (1 << 13)) {
    set_error(WAVEMOTH_ERR_ARG, "invalid Nside");
    return nullptr;
  }
  const int nrings = 4 * Nside - 1;
  char *buf = (char *)malloc(sizeof(wavemoth_grid_info) + sizeof(double) * nrings +
                             sizeof(bfm_index_t) * (nrings + 1));
  if (!buf) return nullptr;
  auto *g = (wavemoth_grid_info *)buf;
  g->phi0s = (double *)(buf + sizeof(wavemoth_grid_info));
  g->ring_offsets = (bfm_index_t *)(g->phi0s + nrings);
  g->has_equator = 1;
  g->nrings = nrings;
  g->mid_ring = 2 * Nside - 1;
  int npr = 0, ipix = 0;
  const double pi = 3.14159265358979323846;
  for (int r = 0; r < nrings; ++r) {
    if (r <= Nside - 1) {
      npr += 4;
      g->phi0s[r] = pi / (4.0 * (r + 1));
    } else if (r > 3 * Nside - 1) {
      npr -= 4;
      g->phi0s[r] = pi / (4.0 * (nrings - r));
    } else {
      g->phi0s[r] = (pi / (4.0 * Nside)) * (r % 2);
    }
    g->ring_offsets[r] = ipix;
    ipix += npr;
  }
  g->ring_offsets[nrings] = ipix;
  g->npix = ipix;
  return g;
}

void wavemoth_free_grid_info(wavemoth_grid_info *info) { free(info); }

}  // extern "C"
