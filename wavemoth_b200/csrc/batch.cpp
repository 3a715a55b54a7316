// Batches of transforms of uneven size executed as one CUDA graph launch.
//
// A batch holds requests (plan, direction, device input, device output) of
// any nside / lmax / number of maps.  At creation the requests are captured
// into one CUDA graph: they are ordered by their algorithmic work (Legendre
// flops plus ring bytes, from wavemoth_plan_work) and assigned longest first
// to the least-loaded of `width` parallel capture branches, so that small
// transforms fill the SMs that large ones leave idle.  A schedule is the
// branch count and, with more than one branch, the number of SMs every
// request's persistent Legendre kernels may occupy (the CTAs that walk its
// (m, parity) tile list; fewer leave room for the concurrent branches).
// Schedules are autotuned: each candidate is captured, instantiated and
// timed, and the fastest is kept (wavemoth_b200.batch caches the choice per
// batch signature).  Every execute is then one cudaGraphLaunch.
//
// Requests of one direction whose plans share a device image (same plan
// file, lmax, precision and settings) are coalesced into one transform of
// their summed map count: the matrices are streamed once for all of them.
// The batch owns that transform's plan (on the same image) and its
// interleaved input and output buffers; inside the graph a copy kernel
// gathers the requests' inputs before it and scatters the outputs after it.
// Every map's arithmetic is independent of the other maps', so the results
// are those of the separate calls.
//
// The plans' own buffers (q, X, operand slices) are shared by all calls on
// one plan, so a batch must not hold two requests on the same plan.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <string>
#include <vector>

#include "kernels.h"
#include "wavemoth.h"
#include "wavemoth_b200.h"

namespace wm {
int set_last_error(int code, const std::string &msg);
bool plans_coalescible(wavemoth_plan a, wavemoth_plan b);
wavemoth_plan plan_with_maps(wavemoth_plan P, int nmaps);
void plan_sizes(wavemoth_plan P, int64_t *nalm, int64_t *npix);
}

struct _wavemoth_batch {
  // a request merged into a coalesced transform: its buffers and its maps'
  // place among the transform's
  struct Member {
    const double *in;
    double *out;
    int nmaps, offset;
  };
  struct Req {
    wavemoth_plan plan;
    int direction;
    const double *in;
    double *out;
    double cost;
    std::vector<Member> members;  // empty: the caller's own request
    double *own_in = nullptr;     // coalesced: the batch's interleaved input
  };
  std::vector<Req> reqs;
  std::vector<wavemoth_plan> owned_plans;
  std::vector<double *> owned_buffers;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int width = 0;
  int sms = 0;  // SMs per request of the chosen schedule (0: all)
  double ms = 0.0;

  ~_wavemoth_batch() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    for (auto p : owned_plans) wavemoth_destroy_plan(p);
    for (auto b : owned_buffers) cudaFree(b);
  }
};

namespace {

int capture_branches(_wavemoth_batch &B, int width, cudaStream_t origin, cudaGraph_t *out);
int run_request(const _wavemoth_batch::Req &r, cudaStream_t st);

int cuda_err(cudaError_t e, const char *what) {
  if (e == cudaSuccess) return 0;
  return wm::set_last_error(WAVEMOTH_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// Captures the batch with `width` branches forked from `origin`, every
// request's persistent Legendre kernels capped at `sms` SMs (launch sizes
// are fixed into the graph; the plans' caps are restored afterwards).
int capture(_wavemoth_batch &B, int width, int sms, cudaStream_t origin, cudaGraph_t *out) {
  for (const auto &r : B.reqs) wavemoth_plan_set_grid_cap(r.plan, width > 1 ? sms : 0);
  const int rc = capture_branches(B, width, origin, out);
  for (const auto &r : B.reqs) wavemoth_plan_set_grid_cap(r.plan, 0);
  return rc;
}

// One request on `st`: a coalesced one gathers its members' inputs (alm
// rows of 2 doubles per map, map rows of 1) into the interleaved buffer,
// runs, and scatters the outputs back.
int run_request(const _wavemoth_batch::Req &r, cudaStream_t st) {
  const bool a2m = r.direction == 0;
  if (r.members.empty())
    return a2m ? wavemoth_execute_alm2map_device(r.plan, r.in, r.out, st)
               : wavemoth_execute_map2alm_device(r.plan, r.in, r.out, st);
  int64_t nalm = 0, npix = 0;
  wm::plan_sizes(r.plan, &nalm, &npix);
  const int64_t ntot = wavemoth_plan_nmaps(r.plan);
  const int64_t in_rows = a2m ? nalm : npix, out_rows = a2m ? npix : nalm;
  const int64_t in_w = a2m ? 2 : 1, out_w = a2m ? 1 : 2;
  int rc = 0;
  for (const auto &m : r.members)
    if (!rc)
      rc = cuda_err(wm::launch_strided_copy(r.own_in + m.offset * in_w, ntot * in_w, m.in, m.nmaps * in_w,
                                            m.nmaps * in_w, in_rows, st), "batch gather");
  if (!rc)
    rc = a2m ? wavemoth_execute_alm2map_device(r.plan, r.in, r.out, st)
             : wavemoth_execute_map2alm_device(r.plan, r.in, r.out, st);
  for (const auto &m : r.members)
    if (!rc)
      rc = cuda_err(wm::launch_strided_copy(m.out, m.nmaps * out_w, r.out + m.offset * out_w, ntot * out_w,
                                            m.nmaps * out_w, out_rows, st), "batch scatter");
  return rc;
}

int capture_branches(_wavemoth_batch &B, int width, cudaStream_t origin, cudaGraph_t *out) {
  std::vector<cudaStream_t> br(width, nullptr);
  std::vector<cudaEvent_t> done(width, nullptr);
  cudaEvent_t fork = nullptr;
  int rc = cuda_err(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming), "batch event");
  for (int i = 0; i < width && !rc; ++i) {
    rc = cuda_err(cudaStreamCreateWithFlags(&br[i], cudaStreamNonBlocking), "batch stream");
    if (!rc) rc = cuda_err(cudaEventCreateWithFlags(&done[i], cudaEventDisableTiming), "batch event");
  }
  bool capturing = false;
  if (!rc) {
    rc = cuda_err(cudaStreamBeginCapture(origin, cudaStreamCaptureModeThreadLocal), "begin capture");
    capturing = !rc;
  }
  if (!rc) rc = cuda_err(cudaEventRecord(fork, origin), "fork");
  for (int i = 0; i < width && !rc; ++i) rc = cuda_err(cudaStreamWaitEvent(br[i], fork, 0), "fork");
  // longest first onto the least-loaded branch
  std::vector<double> load(width, 0.0);
  for (const auto &r : B.reqs) {
    if (rc) break;
    const int b = (int)(std::min_element(load.begin(), load.end()) - load.begin());
    load[b] += r.cost;
    rc = run_request(r, br[b]);
  }
  for (int i = 0; i < width && !rc; ++i) {
    rc = cuda_err(cudaEventRecord(done[i], br[i]), "join");
    if (!rc) rc = cuda_err(cudaStreamWaitEvent(origin, done[i], 0), "join");
  }
  if (capturing) {
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(origin, &g);
    if (!rc) rc = cuda_err(e, "end capture");
    if (rc && g) cudaGraphDestroy(g);
    if (!rc) *out = g;
  }
  for (int i = 0; i < width; ++i) {
    if (br[i]) cudaStreamDestroy(br[i]);
    if (done[i]) cudaEventDestroy(done[i]);
  }
  if (fork) cudaEventDestroy(fork);
  return rc;
}

// Mean time of `reps` launches of an instantiated graph (after one warm-up).
int time_graph(cudaGraphExec_t ex, cudaStream_t st, int reps, double *ms) {
  cudaEvent_t a = nullptr, b = nullptr;
  int rc = cuda_err(cudaEventCreate(&a), "timing event");
  if (!rc) rc = cuda_err(cudaEventCreate(&b), "timing event");
  if (!rc) rc = cuda_err(cudaGraphLaunch(ex, st), "graph launch");
  if (!rc) rc = cuda_err(cudaEventRecord(a, st), "timing event");
  for (int i = 0; i < reps && !rc; ++i) rc = cuda_err(cudaGraphLaunch(ex, st), "graph launch");
  if (!rc) rc = cuda_err(cudaEventRecord(b, st), "timing event");
  if (!rc) rc = cuda_err(cudaEventSynchronize(b), "timing event");
  float t = 0.f;
  if (!rc) rc = cuda_err(cudaEventElapsedTime(&t, a, b), "timing event");
  if (!rc) *ms = t / reps;
  if (a) cudaEventDestroy(a);
  if (b) cudaEventDestroy(b);
  return rc;
}

}  // namespace

namespace {

// Validates the requests, estimates their costs and runs the schedule
// search over `schedules` (pairs of branches, SMs per request).
wavemoth_batch create_batch(int nreq, const wavemoth_plan *plans, const int *directions,
                            const double *const *inputs, double *const *outputs,
                            const std::vector<std::pair<int, int>> &schedules, void *stream) {
  if (nreq <= 0 || !plans || !directions || !inputs || !outputs || schedules.empty()) {
    wm::set_last_error(WAVEMOTH_ERR_ARG, "invalid batch arguments");
    return nullptr;
  }
  auto *B = new _wavemoth_batch();
  for (int i = 0; i < nreq; ++i) {
    if (!plans[i] || !inputs[i] || !outputs[i] || (directions[i] != 0 && directions[i] != 1)) {
      wm::set_last_error(WAVEMOTH_ERR_ARG, "batch request " + std::to_string(i) + " is invalid");
      delete B;
      return nullptr;
    }
    for (int j = 0; j < i; ++j)
      if (plans[j] == plans[i]) {
        wm::set_last_error(WAVEMOTH_ERR_ARG, "two batch requests share one plan (its buffers would race)");
        delete B;
        return nullptr;
      }
  }
  // requests of one direction on one image, in request order
  std::vector<std::vector<int>> groups;
  for (int i = 0; i < nreq; ++i) {
    bool placed = false;
    for (auto &g : groups)
      if (directions[g[0]] == directions[i] && wm::plans_coalescible(plans[g[0]], plans[i])) {
        g.push_back(i);
        placed = true;
        break;
      }
    if (!placed) groups.push_back({i});
  }
  for (const auto &g : groups) {
    _wavemoth_batch::Req r{plans[g[0]], directions[g[0]], inputs[g[0]], outputs[g[0]], 0.0, {}, nullptr};
    if (g.size() > 1) {
      int ntot = 0;
      for (int i : g) {
        r.members.push_back({inputs[i], outputs[i], wavemoth_plan_nmaps(plans[i]), ntot});
        ntot += wavemoth_plan_nmaps(plans[i]);
      }
      r.plan = wm::plan_with_maps(plans[g[0]], ntot);
      if (!r.plan) {
        delete B;
        return nullptr;
      }
      B->owned_plans.push_back(r.plan);
      int64_t nalm = 0, npix = 0;
      wm::plan_sizes(r.plan, &nalm, &npix);
      const int64_t alm_d = 2 * nalm * ntot, map_d = npix * ntot;
      double *in = nullptr, *out = nullptr;
      const bool a2m = r.direction == 0;
      if (cuda_err(cudaMalloc(&in, sizeof(double) * (a2m ? alm_d : map_d)), "batch buffers")) {
        delete B;
        return nullptr;
      }
      B->owned_buffers.push_back(in);
      if (cuda_err(cudaMalloc(&out, sizeof(double) * (a2m ? map_d : alm_d)), "batch buffers")) {
        delete B;
        return nullptr;
      }
      B->owned_buffers.push_back(out);
      r.in = r.own_in = in;
      r.out = out;
    }
    double w[12] = {0};
    if (wavemoth_plan_work(r.plan, wavemoth_plan_nmaps(r.plan), w) != 0) {
      delete B;
      return nullptr;
    }
    // seconds-scale estimate: FP64 flops at 30 TF/s plus ring bytes at 1 TB/s
    r.cost = w[0] / 30e12 + w[3] / 1e12;
    B->reqs.push_back(r);
  }
  std::stable_sort(B->reqs.begin(), B->reqs.end(),
                   [](const _wavemoth_batch::Req &a, const _wavemoth_batch::Req &b) { return a.cost > b.cost; });
  // capture and timing run on a private stream (the legacy default stream
  // cannot be captured); the caller's pending work is waited for first
  cudaStream_t st = nullptr;
  if (cuda_err(cudaStreamSynchronize((cudaStream_t)stream), "batch create") ||
      cuda_err(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "batch stream")) {
    delete B;
    return nullptr;
  }
  const int ntr = (int)B->reqs.size();
  for (const auto &sc : schedules) {
    const int width = std::max(1, std::min(sc.first, ntr)), sms = std::max(0, sc.second);
    cudaGraph_t g = nullptr;
    cudaGraphExec_t ex = nullptr;
    int rc = capture(*B, width, sms, st, &g);
    if (!rc) rc = cuda_err(cudaGraphInstantiate(&ex, g, 0), "graph instantiate");
    double ms = 0.0;
    if (!rc && schedules.size() > 1) rc = time_graph(ex, st, 3, &ms);
    if (rc) {
      if (ex) cudaGraphExecDestroy(ex);
      if (g) cudaGraphDestroy(g);
      cudaStreamDestroy(st);
      delete B;
      return nullptr;
    }
    if (!B->exec || ms < B->ms) {
      if (B->exec) cudaGraphExecDestroy(B->exec);
      if (B->graph) cudaGraphDestroy(B->graph);
      B->exec = ex;
      B->graph = g;
      B->width = width;
      B->sms = width > 1 ? sms : 0;
      B->ms = ms;
    } else {
      cudaGraphExecDestroy(ex);
      cudaGraphDestroy(g);
    }
  }
  cudaStreamSynchronize(st);
  cudaStreamDestroy(st);
  return B;
}

}  // namespace

extern "C" {

wavemoth_batch wavemoth_batch_create(int nreq, const wavemoth_plan *plans, const int *directions,
                                     const double *const *inputs, double *const *outputs, int max_width,
                                     void *stream) {
  // branch counts 1, 2, 4, 8 (up to max_width and the request count), every
  // request on all SMs
  std::vector<std::pair<int, int>> sched;
  const int wmax = std::max(1, std::min(std::min(nreq, 8), max_width > 0 ? max_width : 8));
  for (int width = 1; width <= wmax; width *= 2) sched.push_back({width, 0});
  return create_batch(nreq, plans, directions, inputs, outputs, sched, stream);
}

wavemoth_batch wavemoth_batch_create_scheduled(int nreq, const wavemoth_plan *plans, const int *directions,
                                               const double *const *inputs, double *const *outputs,
                                               const int *schedules, int nschedules, void *stream) {
  if (!schedules || nschedules <= 0) {
    wm::set_last_error(WAVEMOTH_ERR_ARG, "no schedules given");
    return nullptr;
  }
  std::vector<std::pair<int, int>> sched;
  for (int k = 0; k < nschedules; ++k) sched.push_back({schedules[2 * k], schedules[2 * k + 1]});
  return create_batch(nreq, plans, directions, inputs, outputs, sched, stream);
}

int wavemoth_batch_schedule(wavemoth_batch batch, int *width, int *sms, double *ms) {
  if (!batch) return wm::set_last_error(WAVEMOTH_ERR_ARG, "NULL batch");
  if (width) *width = batch->width;
  if (sms) *sms = batch->sms;
  if (ms) *ms = batch->ms;
  return 0;
}

int wavemoth_batch_transforms(wavemoth_batch batch) {
  if (!batch) return wm::set_last_error(WAVEMOTH_ERR_ARG, "NULL batch");
  return (int)batch->reqs.size();
}

int wavemoth_batch_execute(wavemoth_batch batch, void *stream) {
  if (!batch || !batch->exec) return wm::set_last_error(WAVEMOTH_ERR_ARG, "NULL batch");
  return cuda_err(cudaGraphLaunch(batch->exec, (cudaStream_t)stream), "batch launch");
}

int wavemoth_batch_info(wavemoth_batch batch, int *width, double *ms) {
  if (!batch) return wm::set_last_error(WAVEMOTH_ERR_ARG, "NULL batch");
  if (width) *width = batch->width;
  if (ms) *ms = batch->ms;
  return 0;
}

void wavemoth_batch_destroy(wavemoth_batch batch) { delete batch; }

}  // extern "C"
