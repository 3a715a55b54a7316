// The reference's private kernel-level hooks (src/legendre_transform.h:16-38,
// src/butterfly.h.in:141-184), with the same names, arguments and meaning,
// so that its kernel tests can be pointed at this library.
//
// Where a hook computes, it computes on the GPU: the caller's host buffers
// are copied to the device, one of this library's kernels runs and the
// result is copied back.
//   wavemoth_legendre_transform{,_sse}  k_legendre_transform (below): the
//       three-term recurrence and the matrix product of one (m, parity)
//       block, in the reference scalar routine's operation order without
//       contraction (src/legendre_transform.c.in:680-716), so y equals that
//       routine's output bit for bit;
//   bfm_transpose_apply_d               the generic butterfly kernel
//       (legendre.cu) on the serialized matrix, its root rows pulled through
//       the caller's pull function in the reference's order
//       (src/butterfly.c.in:284-432).
// The bookkeeping hooks (_pack, _auxdata, _sse_query_work,
// bfm_query_matrix_data, bfm_scatter, bfm_create_plan) are host code, as in
// the reference: they move or describe data and compute nothing a kernel
// would.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "kernels.h"
#include "plan.h"
#include "program.h"
#include "wavemoth.h"
#include "wavemoth_b200.h"

namespace wm {
int set_last_error(int code, const std::string &msg);  // abi.cpp
}

struct _bfm_plan {
  size_t k_max, nblocks_max, nvecs;
};

namespace {

// Sizes of the reference's SSE packing (src/legendre_transform.c.in:321-327):
// vectors in blocks of 4, rows 2.. in chunks of 4096 / (6 * 8 * 2) = 42.
constexpr size_t kPackNJ = 4;
constexpr size_t kPackKChunk = 4096 / (6 * sizeof(double) * 2);

// One thread per (x, vector): P_k(x) by the recurrence, y = sum_k P_k a_2k.
__global__ void k_legendre_transform(int64_t nx, int64_t nk, int64_t nvecs, const double *__restrict__ a,
                                     double *__restrict__ y, const double *__restrict__ x2,
                                     const double *__restrict__ aux, const double *__restrict__ P0,
                                     const double *__restrict__ P1) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nx * nvecs) return;
  const int64_t i = t / nvecs, j = t % nvecs;
  double pp = P0[i], pc = P1[i];
  double acc = __dmul_rn(pp, a[j]);
  acc = __dadd_rn(acc, __dmul_rn(pc, a[2 * nvecs + j]));
  const double xs = x2[i];
  for (int64_t k = 2; k < nk; ++k) {
    const double *c = aux + 3 * (k - 2);
    const double pv = __dadd_rn(__dmul_rn(__dmul_rn(__dadd_rn(xs, c[0]), c[1]), pc), __dmul_rn(c[2], pp));
    pp = pc;
    pc = pv;
    acc = __dadd_rn(acc, __dmul_rn(pv, a[2 * k * nvecs + j]));
  }
  y[i * nvecs + j] = acc;
}

// Device buffers of one hook call, freed on scope exit.
struct DevBufs {
  std::vector<void *> p;
  ~DevBufs() {
    for (void *q : p) cudaFree(q);
  }
  template <class T>
  T *alloc(size_t n, cudaError_t &e) {
    void *q = nullptr;
    if (e == cudaSuccess) e = cudaMalloc(&q, std::max<size_t>(n, 1) * sizeof(T));
    if (e == cudaSuccess) p.push_back(q);
    return (T *)q;
  }
  template <class T>
  T *upload(const T *src, size_t n, cudaError_t &e) {
    T *d = alloc<T>(n, e);
    if (e == cudaSuccess && n) e = cudaMemcpy(d, src, n * sizeof(T), cudaMemcpyHostToDevice);
    return d;
  }
};

void legendre_transform_device(const char *who, size_t nx, size_t nk, size_t nvecs, const double *a, double *y,
                               const double *x_squared, const double *auxdata, const double *P,
                               const double *Pp1) {
  if (nk < 2 || nvecs == 0) {
    wm::set_last_error(WAVEMOTH_ERR_ARG, std::string(who) + ": need nk >= 2 and nvecs >= 1");
    return;
  }
  if (nx == 0) return;
  cudaError_t e = cudaSuccess;
  DevBufs B;
  const double *da = B.upload(a, (2 * nk - 1) * nvecs, e);
  double *dy = B.alloc<double>(nx * nvecs, e);
  const double *dx = B.upload(x_squared, nx, e);
  const double *daux = B.upload(auxdata, nk > 2 ? 3 * (nk - 2) : 0, e);
  const double *dp0 = B.upload(P, nx, e);
  const double *dp1 = B.upload(Pp1, nx, e);
  if (e == cudaSuccess) {
    const int64_t n = (int64_t)(nx * nvecs);
    k_legendre_transform<<<(unsigned)((n + 127) / 128), 128>>>((int64_t)nx, (int64_t)nk, (int64_t)nvecs, da, dy, dx,
                                                                daux, dp0, dp1);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(y, dy, nx * nvecs * sizeof(double), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) wm::set_last_error(WAVEMOTH_ERR_CUDA, std::string(who) + ": " + cudaGetErrorString(e));
}

// The reference's packer over rows [0, nk) of `plain` (row k at 2 k nvecs):
// chunks of kPackKChunk rows, within a chunk vector blocks of kPackNJ, within
// a block row after row (src/legendre_transform.c.in:330-363).  unpack = the
// inverse copy.
void pack_rows(size_t nk, size_t nvecs, const double *plain, double *packed, bool unpack, size_t &pos) {
  for (size_t k0 = 0; k0 < nk; k0 += kPackKChunk) {
    const size_t k1 = std::min(nk, k0 + kPackKChunk);
    const size_t jfull = nvecs - nvecs % kPackNJ;
    auto move = [&](size_t k, size_t j, size_t n) {
      double *pl = const_cast<double *>(plain) + 2 * k * nvecs + j;
      if (unpack) memcpy(pl, packed + pos, n * sizeof(double));
      else memcpy(packed + pos, pl, n * sizeof(double));
      pos += n;
    };
    for (size_t j0 = 0; j0 < jfull; j0 += kPackNJ)
      for (size_t k = k0; k < k1; ++k) move(k, j0, kPackNJ);
    if (jfull < nvecs)
      for (size_t k = k0; k < k1; ++k) move(k, jfull, nvecs - jfull);
  }
}

}  // namespace

extern "C" {

void wavemoth_legendre_transform(size_t nx, size_t nk, size_t nvecs, double *a_l, double *y, double *x_squared,
                                 double *auxdata, double *P, double *Pp1) {
  legendre_transform_device("wavemoth_legendre_transform", nx, nk, nvecs, a_l, y, x_squared, auxdata, P, Pp1);
}

void wavemoth_legendre_transform_sse(size_t nx, size_t nk, size_t nvecs, double *a_l, double *y,
                                     double *x_squared, double *auxdata, double *P, double *Pp1, char *work) {
  (void)work;
  if (nvecs % 2 != 0 || nk < 2) {
    wm::set_last_error(WAVEMOTH_ERR_ARG, "wavemoth_legendre_transform_sse: nvecs must be even and nk >= 2");
    return;
  }
  // a_l is in the packed layout of wavemoth_legendre_transform_pack
  std::vector<double> plain((2 * nk - 1) * nvecs, 0.0);
  if (nvecs == 2) {
    for (size_t k = 0; k < nk; ++k) {
      plain[4 * k] = a_l[2 * k];
      plain[4 * k + 1] = a_l[2 * k + 1];
    }
  } else {
    size_t pos = 0;
    pack_rows(2, nvecs, plain.data(), a_l, true, pos);
    pack_rows(nk - 2, nvecs, plain.data() + 4 * nvecs, a_l, true, pos);
  }
  legendre_transform_device("wavemoth_legendre_transform_sse", nx, nk, nvecs, plain.data(), y, x_squared, auxdata,
                            P, Pp1);
}

size_t wavemoth_legendre_transform_sse_query_work(size_t nvecs) {
  // the reference's sizes (src/legendre_transform.c.in:625-633); the device
  // routine itself needs no work buffer
  // (the reference's chunk macro is unparenthesised, so its product
  // evaluates as (nvecs * 4096) / 96 * 8 in integer arithmetic)
  if (nvecs == 2) return 0;
  return std::max<size_t>(4096, nvecs * 4096 / (6 * sizeof(double) * 2) * sizeof(double));
}

void wavemoth_legendre_transform_pack(size_t nk, size_t nvecs, double *input, double *output) {
  if (nk < 2 || nvecs % 2 != 0) {
    wm::set_last_error(WAVEMOTH_ERR_ARG, "wavemoth_legendre_transform_pack: need nk >= 2 and even nvecs");
    return;
  }
  if (nvecs == 2) {
    for (size_t k = 0; k < nk; ++k) {
      output[2 * k] = input[4 * k];
      output[2 * k + 1] = input[4 * k + 1];
    }
    return;
  }
  size_t pos = 0;
  pack_rows(2, nvecs, input, output, false, pos);
  pack_rows(nk - 2, nvecs, input + 4 * nvecs, output, false, pos);
}

void wavemoth_legendre_transform_auxdata(size_t m, size_t lmin, size_t nk, double *auxdata) {
  // alpha = -d_{l-2}, beta = 1 / c_{l-2}, gamma = -c_{l-4} / c_{l-2} for l =
  // lmin + 2k, k >= 2, with c and d of src/legendre_transform.c.in:723-747
  // (integer products as there, in size_t arithmetic)
  double cp = 0.0, cpp = 0.0, dp = 0.0;
  for (size_t k = 0, l = lmin; k < nk; ++k, l += 2) {
    const double cx = (double)((l - m + 1) * (l - m + 2) * (l + m + 1) * (l + m + 2));
    const double cy = (double)((2 * l + 1) * (2 * l + 3) * (2 * l + 3) * (2 * l + 5));
    const double c = sqrt(cx / cy);
    const double dx = (double)(2 * l * (l + 1) - 2 * m * m - 1);
    const double dy = (double)((2 * l - 1) * (2 * l + 3));
    const double d = dx / dy;
    if (k >= 2) {
      auxdata[3 * (k - 2)] = -dp;
      auxdata[3 * (k - 2) + 1] = 1 / cp;
      auxdata[3 * (k - 2) + 2] = -cpp / cp;
    }
    dp = d;
    cpp = cp;
    cp = c;
  }
}

char *bfm_query_matrix_data(char *head, bfm_matrix_data_info *info) {
  int32_t h[4], t[4];
  int64_t ec;
  memcpy(h, head, 16);
  memcpy(&ec, head + 16, 8);
  memcpy(t, head + 24, 16);
  info->nrows = (size_t)h[0];
  info->ncols = (size_t)h[1];
  info->k_max = (size_t)h[2];
  info->nblocks_max = (size_t)h[3];
  info->element_count = (size_t)ec;
  info->first_level_size = (size_t)t[0];
  info->heap_size = (size_t)t[1];
  info->heap_first_index = (size_t)t[2];
  return head + 40;
}

const char *bfm_scatter(const char *mask, double *target1, double *target2, const double *source, size_t len1,
                        size_t len2, size_t nvecs, int group, int should_add) {
  // rows of `source` whose mask entry equals `group` go, in order, to the
  // rows of target1 (first len1 mask entries) and target2 (next len2)
  // (src/butterfly.c.in:57-139); other target rows are left alone
  if ((group != 0 && group != 1) || nvecs % 2 != 0) {
    wm::set_last_error(WAVEMOTH_ERR_ARG, "bfm_scatter: invalid group or odd nvecs");
    return nullptr;
  }
  double *tgt[2] = {target1, target2};
  const size_t len[2] = {len1, len2};
  for (int t = 0; t < 2; ++t)
    for (size_t r = 0; r < len[t]; ++r, ++mask) {
      if (*mask == group) {
        for (size_t v = 0; v < nvecs; ++v) tgt[t][v] = should_add ? tgt[t][v] + source[v] : source[v];
        source += nvecs;
      }
      tgt[t] += nvecs;
    }
  return mask;
}

bfm_plan *bfm_create_plan(size_t k_max, size_t nblocks_max, size_t nvecs, void *mem_semaphore,
                          void *cpu_semaphore) {
  (void)mem_semaphore;
  (void)cpu_semaphore;
  if (nvecs == 0) {
    wm::set_last_error(WAVEMOTH_ERR_ARG, "bfm_create_plan: nvecs must be positive");
    return nullptr;
  }
  return new _bfm_plan{k_max, nblocks_max, nvecs};
}

void bfm_destroy_plan(bfm_plan *plan) { delete plan; }

int bfm_transpose_apply_d(bfm_plan *plan, char *matrix_data, pull_func_t pull_func, double *target,
                          size_t target_len, void *caller_ctx) {
  if (!plan || !matrix_data || !pull_func || !target)
    return wm::set_last_error(WAVEMOTH_ERR_ARG, "bfm_transpose_apply_d: NULL argument");
  if ((uintptr_t)matrix_data % 16 != 0)
    return wm::set_last_error(WAVEMOTH_ERR_ARG, "bfm_transpose_apply_d: matrix_data not 16-byte aligned");
  bfm_matrix_data_info info;
  bfm_query_matrix_data(matrix_data, &info);
  const size_t nvecs = plan->nvecs;
  if (target_len != nvecs * info.ncols)
    return wm::set_last_error(WAVEMOTH_ERR_ARG, "bfm_transpose_apply_d: target_len does not match ncols * nvecs");
  // like the reference, the matrix data is trusted to hold what its tables
  // point to; its extent is not known here
  wm::HostProgram P;
  std::string err;
  if (!wm::compile_butterfly_tree(matrix_data, (size_t)1 << 40, P, err))
    return wm::set_last_error(WAVEMOTH_ERR_RESOURCE, "bfm_transpose_apply_d: " + err);
  const wm::DevMatrix &M = P.mats[0];
  const size_t nroots = info.first_level_size;
  // residual payload table of root r: int64 n, then n + 1 offsets from the
  // matrix start (src/butterfly.c.in:311-316)
  auto payloads = [&](size_t r, std::vector<int64_t> &po) {
    int64_t toff;
    memcpy(&toff, matrix_data + 40 + 8 * r, 8);
    int64_t n;
    memcpy(&n, matrix_data + toff, 8);
    po.resize((size_t)n + 1);
    memcpy(po.data(), matrix_data + toff + 8, 8 * ((size_t)n + 1));
  };
  std::vector<int64_t> po;
  if (M.nlevels == 0) {
    // leaf roots stream straight to the target (src/butterfly.c.in:303-309)
    size_t start = 0;
    for (size_t r = 0; r < nroots; ++r) {
      payloads(r, po);
      int32_t n;
      int64_t hoff;
      memcpy(&hoff, matrix_data + 40 + 8 * (nroots + r), 8);
      memcpy(&n, matrix_data + hoff + 4, 4);
      pull_func(target, start, start + (size_t)n, nvecs, matrix_data + po[0], (size_t)(po[1] - po[0]), caller_ctx);
      start += (size_t)n;
    }
    return 0;
  }
  // root rows, pulled block after block (heap order, then (T, B) of every
  // pair) into the depth-0 buffer of the compiled tree
  std::vector<double> h0((size_t)M.root_rows * nvecs, 0.0);
  {
    const wm::DevLevel &L0 = P.levels[M.level_begin];
    int32_t pair = L0.pair_begin;
    for (size_t r = 0; r < nroots; ++r) {
      payloads(r, po);
      int64_t hoff;
      memcpy(&hoff, matrix_data + 40 + 8 * (nroots + r), 8);
      int32_t nblocks;
      memcpy(&nblocks, matrix_data + hoff, 4);
      size_t input_pos = 0;
      for (int32_t b = 0; b < nblocks; ++b, pair += (b % 2 == 0)) {
        const wm::DevPair &pr = P.pairs[pair];
        const int32_t k = (b % 2 == 0) ? pr.kT : pr.kB;
        const int32_t row = (b % 2 == 0) ? pr.inT : pr.inB;
        pull_func(h0.data() + (size_t)row * nvecs, input_pos, input_pos + (size_t)k, nvecs, matrix_data + po[b],
                  (size_t)(po[b + 1] - po[b]), caller_ctx);
        input_pos += (size_t)k;
      }
    }
  }
  cudaError_t e = cudaSuccess;
  DevBufs B;
  const int64_t slot = 2 * (int64_t)std::max<int32_t>(M.max_rows, 1) * (int64_t)nvecs;
  double *scratch = B.alloc<double>((size_t)slot, e);
  if (e == cudaSuccess) e = cudaMemcpy(scratch, h0.data(), h0.size() * sizeof(double), cudaMemcpyHostToDevice);
  const int32_t zero = 0;
  wm::LegendreParams p{};
  p.mats = B.upload(P.mats.data(), P.mats.size(), e);
  p.levels = B.upload(P.levels.data(), P.levels.size(), e);
  p.pairs = B.upload(P.pairs.data(), P.pairs.size(), e);
  p.f64 = B.upload(P.f64.data(), P.f64.size(), e);
  p.i32 = B.upload(P.i32.data(), P.i32.size(), e);
  p.order = B.upload(&zero, 1, e);
  p.counter = B.upload(&zero, 1, e);
  double *dt = B.alloc<double>(target_len, e);
  if (e == cudaSuccess) {
    p.nmats = 1;
    p.lmax = 0;
    p.nvecs = (int32_t)nvecs;
    p.q_out = dt;
    p.q_mstride = 0;
    p.q_rstride = (int64_t)nvecs;
    p.scratch = scratch;
    p.slot_stride = slot;
    p.level0_given = 1;
    e = wm::launch_legendre(true, p, 1, 0);
  }
  if (e == cudaSuccess) e = cudaMemcpy(target, dt, target_len * sizeof(double), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess)
    return wm::set_last_error(WAVEMOTH_ERR_CUDA, std::string("bfm_transpose_apply_d: ") + cudaGetErrorString(e));
  return 0;
}

}  // extern "C"
