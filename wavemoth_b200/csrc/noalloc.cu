// Allocation-free entry point for the alm2map Legendre step.
//
// Some callers cannot call cudaMalloc at the moment they run the transform:
// code inside a custom allocator's callback, a process whose memory is
// managed by a framework that forbids outside allocations, or a step that
// must not trigger driver allocations while other work is latency
// critical.  wavemoth_legendre_alm2map_noalloc runs the generic FP64
// butterfly Legendre kernel (k_alm2map_legendre, SIMT, persistent CTAs on a
// work queue) over every (m, parity) matrix of the plan; the plan's own path
// runs that kernel only for trees of depth >= 2 and the FP64 tensor-core
// kernels for the rest, so the two agree to rounding, not bitwise.  Its
// per-CTA level buffers and its work-queue counter come from the
// file-scope device array below instead of plan-allocated scratch.  The
// caller passes the input (alm) and the output (q) as device pointers; the
// plan (created beforehand) supplies the compiled butterfly program.
//
// The array is a fixed 32 MiB that every GPU which loads the library holds
// until the process exits.  Its device address is resolved when a plan is
// created on a device (abi.cpp), which loads the module holding it: that is
// when the 32 MiB are taken, and the kernel's module is loaded then too, so
// the call itself makes the driver allocate nothing.  All calls share the
// array, so calls that overlap on the GPU (on different streams, or from
// different host threads) race on it; serialise them.  The counter at its
// start is cleared on every call.
#include <cuda_runtime.h>
#include <stdint.h>

#include <stdio.h>

#include <algorithm>
#include <mutex>
#include <string>

#include "kernels.h"
#include "plan.h"
#include "wavemoth.h"
#include "wavemoth_b200.h"

namespace wm {
// defined in abi.cpp
int set_last_error(int code, const std::string &msg);
bool plan_legendre_params(wavemoth_plan plan, LegendreParams &p, int &grid, std::string &err);
}  // namespace wm

namespace {

constexpr size_t kStaticScratchBytes = size_t(32) << 20;   // 32 MiB
constexpr size_t kCounterBytes = 256;                       // first 256 bytes: counter

__device__ __align__(256) unsigned char g_noalloc_scratch[kStaticScratchBytes];

constexpr int kMaxDevices = 64;
void *g_scratch_addr[kMaxDevices] = {};
std::mutex g_scratch_mutex;

}  // namespace

namespace wm {

// Device address of g_noalloc_scratch on the current device, looked up once
// per device with that device current.  In host code the symbol itself is
// only a host-side stand-in, never a device address.
int noalloc_scratch(void **out, size_t *bytes, std::string &err) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    err = std::string("cudaGetDevice: ") + cudaGetErrorString(e);
    return -1;
  }
  if (dev < 0 || dev >= kMaxDevices) {
    err = "device ordinal out of range for the static scratch table";
    return -1;
  }
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  if (!g_scratch_addr[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) {
      err = std::string("cudaGetSymbolAddress(static scratch): ") + cudaGetErrorString(e);
      return -1;
    }
    g_scratch_addr[dev] = p;
  }
  *out = g_scratch_addr[dev];
  *bytes = kStaticScratchBytes;
  return 0;
}

}  // namespace wm

extern "C" int wavemoth_legendre_alm2map_noalloc(wavemoth_plan plan, const double *alm, double *q,
                                                 void *stream) {
  if (!plan || !alm || !q) return wm::set_last_error(WAVEMOTH_ERR_ARG, "NULL plan or buffer");
  std::string err;
  wm::LegendreParams p{};
  int grid = 0;
  if (!wm::plan_legendre_params(plan, p, grid, err)) return wm::set_last_error(WAVEMOTH_ERR_ARG, err);
  void *base = nullptr;
  size_t bytes = 0;
  if (wm::noalloc_scratch(&base, &bytes, err)) return wm::set_last_error(WAVEMOTH_ERR_CUDA, err);
  const size_t slot_bytes = (size_t)p.slot_stride * sizeof(double);
  const size_t slots_fit = (bytes - kCounterBytes) / slot_bytes;
  if (slots_fit < 1) {
    char msg[256];
    snprintf(msg, sizeof msg,
             "wavemoth_legendre_alm2map_noalloc: one CTA needs %zu bytes of level buffers "
             "(2 x %lld rows x %d vectors), more than the %zu-byte static scratch",
             slot_bytes, (long long)(p.slot_stride / (2 * p.nvecs)), p.nvecs, bytes - kCounterBytes);
    return wm::set_last_error(WAVEMOTH_ERR_NOMEM, msg);
  }
  const int nslots = (int)std::min<size_t>((size_t)grid, slots_fit);
  cudaStream_t st = (cudaStream_t)stream;
  p.counter = (int32_t *)base;
  p.scratch = (double *)((unsigned char *)base + kCounterBytes);
  p.alm_in = alm;
  p.q_out = q;
  // the caller's q is in the layout of wavemoth_get_work: row (2m + parity) ni + ring
  p.q_mstride = (int64_t)p.ni * p.nvecs;
  p.q_rstride = p.nvecs;
  cudaError_t e = cudaMemsetAsync(base, 0, sizeof(int32_t), st);
  if (e == cudaSuccess) e = wm::launch_legendre(true, p, nslots, st);
  if (e != cudaSuccess)
    return wm::set_last_error(WAVEMOTH_ERR_CUDA,
                              std::string("wavemoth_legendre_alm2map_noalloc: ") + cudaGetErrorString(e));
  return 0;
}
