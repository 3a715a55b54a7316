"""Benchmark: alm2map + map2alm round trips on HEALPix, maps per second.

Workload (default): nside 1024, lmax = mmax = 2048, 32 maps per step; alm
re/im iid N(0,1)(l+1)^-1 (Im = 0 at m = 0), one seeded generator per map;
the butterfly plan file is written by wavemoth_b200.resource (ID eps 1e-10,
chunk 64, memop cost 20) into the plan cache before anything is timed.
A step = alm2map of the batch followed by map2alm of the resulting maps.

Contract: ``python bench.py --gpus N --steps K --warmup W``; N > 1 runs
under torch.distributed.run with one rank per GPU, each rank processing its
own batch of maps (weak scaling, no data-path collective: the maps of a batch
are independent).  Rank 0 prints one JSON line.  ``--impl reference`` times
the reference's own C implementation (oracle/_ref) on the host cores instead.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "alm2map+map2alm maps/sec nside=1024 lmax=2048: batched/split vs plain FP64 at ≤1e-9"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--nside", type=int, default=1024)
    ap.add_argument("--lmax", type=int, default=None)
    ap.add_argument("--nmaps", type=int, default=32)
    ap.add_argument("--eps", type=float, default=1e-10)
    ap.add_argument("--chunk", type=int, default=64)
    ap.add_argument("--memop", type=float, default=20.0)
    ap.add_argument("--max-levels", type=int, default=1,
                    help="cap on the interpolation levels of the plan files this script writes: 1 keeps "
                         "every matrix on the tensor-core paths (trees of depth 0 and 1); -1: the "
                         "writer's cost model over all levels")
    ap.add_argument("--plan-dir", default=os.environ.get("WAVEMOTH_PLAN_DIR",
                                                         os.path.join(ROOT, ".plan_cache")))
    ap.add_argument("--cpu-baseline-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=64,
                    help="minimum steps of the end-to-end (host buffers) run: a stream of batches, "
                         "whose first upload and last download (about 19 ms each at nside 1024, 32 maps) "
                         "overlap no transform")
    ap.add_argument("--precision", default="split", choices=["split", "double"],
                    help="split: sliced int8 tensor-core residual products (the plain FP64 path "
                         "is timed beside it and is the error reference); double: plain FP64 only")
    ap.add_argument("--uneven", action="store_true",
                    help="uneven batch instead of the headline workload: --requests seeded requests "
                         "(nside from --uneven-nsides, lmax = 2 nside, 1-8 maps, split alm2map) as one "
                         "graph launch, against the same requests called one after another")
    ap.add_argument("--compare-dense", action="store_true",
                    help="round-trip maps/s of dense-recurrence plans (no butterfly file) against "
                         "butterfly plans at each of --dense-nsides (lmax = 2 nside), both precisions")
    ap.add_argument("--dense-nsides", default="32,64,128,256,512")
    ap.add_argument("--requests", type=int, default=24)
    ap.add_argument("--uneven-nsides", default="128,256,512,1024,2048")
    ap.add_argument("--max-nside2048", type=int, default=1,
                    help="uneven batch: at most this many nside 2048 requests (later such draws are "
                         "drawn again from the other nsides), so that the batch fits one GPU")
    ap.add_argument("--schedule-cache", default=None,
                    help="batch schedule cache (JSON); default a fresh file, so the search runs")
    ap.add_argument("--no-parity", action="store_true",
                    help="skip the comparison of maps 0-3 with the reference's own C alm2map "
                         "(run outside the timed region, rank 0 at N = 1)")
    a = ap.parse_args()
    if a.lmax is None:
        a.lmax = 2 * a.nside
    return a


def log(*args):
    print(*args, file=sys.stderr, flush=True)


# --------------------------------------------------------------------- plan

def plan_levels(a):
    lv = getattr(a, "max_levels", None)
    return None if lv is None or lv < 0 else lv


def plan_path(a):
    lv = "" if plan_levels(a) is None else "_levels%d" % plan_levels(a)
    return os.path.join(a.plan_dir, "rev1_nside%d_lmax%d_eps%g_chunk%d_memop%g%s.dat"
                        % (a.nside, a.lmax, a.eps, a.chunk, a.memop, lv))


def ensure_plan(a, rank):
    from wavemoth_b200 import resource
    path = plan_path(a)
    if os.path.exists(path):
        return path
    if rank == 0:
        os.makedirs(a.plan_dir, exist_ok=True)
        t = time.time()
        log("writing plan file %s ..." % path)
        resource.compute_resource_file(path, a.nside, a.lmax, chunk_size=a.chunk, eps=a.eps,
                                       memop_cost=a.memop, max_levels=plan_levels(a))
        log("plan written in %.1f s" % (time.time() - t))
        return path
    deadline = time.time() + 1800
    while not os.path.exists(path):
        if time.time() > deadline:
            raise TimeoutError("rank %d: plan file never appeared" % rank)
        time.sleep(2)
    return path


def synthetic_alm(lmax, nmaps, seed0, power=1.0):
    """complex128 (nalm, nmaps); map k uses its own generator seeded seed0 + k."""
    ls = np.concatenate([np.arange(m, lmax + 1) for m in range(lmax + 1)])
    ms = np.concatenate([np.full(lmax - m + 1, m) for m in range(lmax + 1)])
    scale = (ls + 1.0) ** -power
    out = np.empty((ls.shape[0], nmaps), np.complex128)
    for k in range(nmaps):
        g = np.random.default_rng(seed0 + k)
        re = g.standard_normal(ls.shape[0])
        im = g.standard_normal(ls.shape[0])
        im[ms == 0] = 0.0
        out[:, k] = (re + 1j * im) * scale
    return out


def rank_seed(rank, nmaps):
    """First generator seed of a rank's batch: the ranks' maps are disjoint."""
    return 1000 + rank * nmaps


def reduce_max_seconds(t, dist=None, device="cuda"):
    """Slowest rank's time (the job's time)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return t
    import torch
    x = torch.tensor([t], dtype=torch.float64, device=device)
    dist.all_reduce(x, op=dist.ReduceOp.MAX)
    return float(x.item())


def job_rate(world, nmaps, steps, seconds):
    """Whole-job maps per second: every rank's maps over the slowest time."""
    return world * nmaps * steps / seconds


# ------------------------------------------------------------------- clocks

class ClockSampler:
    """nvidia-smi clocks/throttle sampling while the timed region runs."""
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.QUERY,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i] == "Active"})
        loaded = [s for s in sm if smax and s > 0.5 * max(smax)] or sm
        return {"sm_mhz": statistics.median(loaded) if loaded else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": reasons,
                "samples": len(rows)}


# ------------------------------------------------------------ CPU baseline

_REF_WORKER = {}


def _ref_worker_init(nside, lmax, nmaps, path, threads, seed0):
    """Pool worker: one reference plan of `threads` threads (a process of its
    own: the reference's plan code is reliable with at most 8 threads, one
    per presented NUMA node)."""
    from oracle import ref
    with ref.stdout_to_stderr():
        rp = ref.RefPlan(nside, lmax, nmaps, path, nthreads=threads)
    rp.input[:] = synthetic_alm(lmax, nmaps, seed0)
    _REF_WORKER["rp"] = rp


def _ref_worker_run(what):
    rp = _REF_WORKER["rp"]
    t0 = time.perf_counter()
    if what == "legendre":
        rp.perform_legendre_transforms()
    else:
        rp.execute()
    return time.perf_counter() - t0


class ReferenceRunner:
    """The reference's own C alm2map (oracle/_ref, built from its sources)
    on the host cores: the first plan in this process (maps 0-3, the
    parity sample) and, to use every core, further independent plans in
    worker processes (spawned), each with 8 threads (its plan code runs
    reliably with at most one thread per presented NUMA node, at most 8).
    A step runs every plan's execute at once; the rate is all plans' maps
    over the wall time.  The reference has no map2alm; a round trip is
    costed as two alm2map executes (the adjoint performs the same
    multiply-adds over the same compressed matrices)."""

    def __init__(self, a, path, nmaps=4, all_cores=True):
        from oracle import ref
        self.nmaps = nmaps
        cores = len(os.sched_getaffinity(0))
        self.threads = max(1, min(ref.MAX_THREADS, cores))
        with ref.stdout_to_stderr():
            self.rp = ref.RefPlan(a.nside, a.lmax, nmaps, path, nthreads=self.threads)
        self.rp.input[:] = synthetic_alm(a.lmax, nmaps, 1000)
        self.extra = max(0, cores // self.threads - 1) if all_cores else 0
        self.pool = None
        if self.extra:
            import multiprocessing as mp
            self.pool = mp.get_context("spawn").Pool(
                self.extra, initializer=_ref_worker_init,
                initargs=(a.nside, a.lmax, nmaps, path, self.threads, 2000))

    def _run(self, what):
        t0 = time.perf_counter()
        pending = self.pool.map_async(_ref_worker_run, [what] * self.extra) if self.pool else None
        if what == "legendre":
            self.rp.perform_legendre_transforms()
        else:
            self.rp.execute()
        if pending is not None:
            pending.get()
        return time.perf_counter() - t0

    def execute(self):
        return self._run("execute")

    def legendre(self):
        return self._run("legendre")

    @property
    def plans(self):
        return 1 + self.extra

    def rate(self, t):
        return self.plans * self.nmaps / (2.0 * t)

    def describe(self, n):
        return ("reference C alm2map (wavemoth_execute; FFT through the oracle's shim, not "
                "FFTW), %d plan(s) of %d maps and %d thread(s) running at once (%d cores); best of "
                "%d steps after warm-up; round trip costed as 2 alm2map (the reference has no map2alm)"
                % (self.plans, self.nmaps, self.threads, self.plans * self.threads, n))

    def close(self):
        self.rp.close()
        if self.pool is not None:
            self.pool.close()
            self.pool.join()
            self.pool = None


def map2alm_restatement_rate(a, path, seconds):
    """map2alm on the host: the reference has none, so this times the
    oracle's FP64 restatement (numpy FFT per ring, butterfly transposed
    applies of the same plan file) on one map, over the m values it reaches
    in `seconds` (every step-th m), scaled to all m by their Legendre
    elements.  One thread (numpy)."""
    from oracle import sht as osht
    f = osht.Rev1File(path)
    npix = 12 * a.nside * a.nside
    maps = np.random.default_rng(5).standard_normal((npix, 1))
    t0 = time.perf_counter()
    work = osht.forward_ffts(maps, a.nside, a.lmax)
    t_fft = time.perf_counter() - t0
    step = max(1, (a.lmax + 1) // 64)
    done_elems, t_leg = 0, 0.0
    total = sum(a.lmax - m + 1 for m in range(a.lmax + 1))
    for m in range(0, a.lmax + 1, step):
        t1 = time.perf_counter()
        for odd in (0, 1):
            mat = f.matrix(m, odd)
            nk = max(0, (a.lmax - m - odd) // 2 + 1)
            if mat is not None and nk:
                mat.apply(np.ascontiguousarray(work[m, odd]).view(np.float64).reshape(2 * a.nside, 2), nk)
        t_leg += time.perf_counter() - t1
        done_elems += a.lmax - m + 1
        if t_fft + t_leg > seconds:
            break
    t_full = t_fft + t_leg * total / max(done_elems, 1)
    return {"value": 1.0 / t_full, "unit": "maps/s (map2alm only)", "cores": 1, "kind": "port",
            "sample": "oracle restatement (numpy FFT + butterfly transposed applies of the same plan "
                      "file), 1 map; Legendre timed over %d elements of %d and scaled" % (done_elems, total)}


def reference_rate(a, path, seconds, runner=None):
    r = runner if runner is not None else ReferenceRunner(a, path)
    r.execute()  # warm-up: page-in and first touch
    times = []
    t_end = time.time() + seconds
    while True:
        times.append(r.execute())
        if time.time() > t_end:
            break
    best = min(times)
    leg = min(r.legendre() for _ in range(3))
    out = {"value": r.rate(best), "unit": "maps/s", "cores": r.threads * r.plans, "kind": "reference",
           "sample": r.describe(len(times)), "seconds_per_execute": best,
           "legendre_phase": {"value": r.plans * r.nmaps / leg, "unit": "maps/s (alm2map Legendre phase "
                              "only, wavemoth_perform_legendre_transforms: shbench -F)",
                              "seconds_per_call": leg}}
    r.close()
    return out


# --------------------------------------------------------------- GPU arm

def fp64_peak_tflops(torch):
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e9
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1) / 1e3)
    del a, b
    return 2.0 * n ** 3 / best / 1e12


def int8_peak_tops(torch):
    """Dense int8 tensor throughput of this GPU (cuBLASLt through
    torch._int_mm, 8192^3), or None if unavailable."""
    try:
        n = 8192
        a = torch.randint(-64, 64, (n, n), dtype=torch.int8, device="cuda")
        b = torch.randint(-64, 64, (n, n), dtype=torch.int8, device="cuda")
        torch._int_mm(a, b)
        torch.cuda.synchronize()
        best = 1e9
        for _ in range(5):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            torch._int_mm(a, b)
            e1.record()
            e1.synchronize()
            best = min(best, e0.elapsed_time(e1) / 1e3)
        del a, b
        return 2.0 * n ** 3 / best / 1e12
    except Exception:
        return None


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d.get("hbm_gbs"), "measured"
    return 6650.0, "fallback"


def measured_peaks_bf16():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d.get("bf16_tflops", 1590.0))
    return 1590.0


def profile_traffic(kernel):
    """DRAM bytes per launch from a committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f).get(kernel)
    return None


def adjoint_identity(torch, T, alm, maps, npix, seed=7):
    """map2alm pinned through the adjoint identity on every map of the batch:
    <alm2map(a), f> = (npix / 4 pi) sum_lm c_m Re(a_lm conj(map2alm(f)_lm))
    (c_0 = 1, c_m = 2) for a seeded Gaussian map f; returns the largest
    |lhs - rhs| / (|alm2map(a)| |f|) over the maps."""
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    f = torch.randn(maps.shape, dtype=torch.float64, device="cuda", generator=g)
    b = T.map2alm(f)
    lmax = T.lmax
    w = torch.cat([torch.full((lmax - m + 1,), 1.0 if m == 0 else 2.0, dtype=torch.float64)
                   for m in range(lmax + 1)]).cuda()
    lhs = (maps * f).sum(0)
    rhs = (w[:, None] * (alm * b.conj()).real).sum(0) * (npix / (4 * np.pi))
    den = maps.norm(dim=0) * f.norm(dim=0)
    return float(((lhs - rhs).abs() / den).max())


def headline_parity(runner, head, nmaps):
    """Maps 0-3 of the GPU batch against the reference's own alm2map of the
    same seeded alm: max |gpu - ref| / max |ref| and the relative L2 error."""
    ref = runner.rp.execute().copy()
    k = min(ref.shape[1], nmaps)
    out = {"reference": "reference C wavemoth_execute (oracle/_ref) on the same plan file, maps 0-%d"
                        % (k - 1)}
    for name in ("plain", "double", "split"):
        if name not in head:
            continue
        got = head[name][:, :k]
        key = "plain" if name == "double" else name
        out[key] = {"max_rel_error_map": float(np.abs(got - ref[:, :k]).max() / np.abs(ref[:, :k]).max()),
                    "rel_l2_error_map": float(np.linalg.norm(got - ref[:, :k]) / np.linalg.norm(ref[:, :k]))}
    return out


def run_b200(a):
    import torch
    import torch.distributed as dist
    from wavemoth_b200.sht import Transform

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    path = ensure_plan(a, rank)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))

    def barrier():
        if world > 1:
            dist.barrier()

    t0 = time.time()
    T = Transform(path, a.nside, a.lmax, a.nmaps, precision=a.precision)
    log("plan loaded in %.1f s" % (time.time() - t0))
    work = T.work()
    alm_h = synthetic_alm(a.lmax, a.nmaps, rank_seed(rank, a.nmaps))
    alm = torch.from_numpy(alm_h).cuda()
    maps = torch.empty((T.npix, a.nmaps), dtype=torch.float64, device="cuda")
    alm_out = torch.empty_like(alm)

    def step(src):
        T.alm2map(src, out=maps)
        T.map2alm(maps, out=alm_out)

    # plain FP64 path beside the split one: its rate and the split error
    plain = None
    head = {}  # maps 0-3 of both paths, compared with the reference after the timed region
    if a.precision == "split":
        TP = Transform(path, a.nside, a.lmax, a.nmaps, precision="double")
        maps_p = torch.empty_like(maps)
        alm_p = torch.empty_like(alm)

        def step_p(src):
            TP.alm2map(src, out=maps_p)
            TP.map2alm(maps_p, out=alm_p)

        for _ in range(a.warmup):
            step_p(alm)
        torch.cuda.synchronize()
        barrier()
        TP.timing(1)
        p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        p0.record()
        for _ in range(a.steps):
            step_p(alm)
        p1.record()
        torch.cuda.synchronize()
        pkt = TP.timing(2)
        TP.timing(0)
        pms = 1e3 * reduce_max_seconds(p0.elapsed_time(p1) / 1e3, dist if world > 1 else None)
        step(alm)
        torch.cuda.synchronize()
        T.device_status()

        def maxrel(x, y):
            return float((x - y).abs().max() / y.abs().max())

        plain = {"value": job_rate(world, a.nmaps, a.steps, pms / 1e3), "unit": "maps/s",
                 "ms_per_step": pms / a.steps,
                 "max_rel_error_map": maxrel(maps, maps_p),
                 "max_rel_error_alm_round_trip": maxrel(alm_out, alm_p),
                 "error_definition": "max |split - plain FP64| / max |plain FP64| over the alm2map "
                                     "output and over the alm2map+map2alm output, same inputs"}
        # the plain path's FP64 tensor-core Legendre phases against DGEMM
        fp64_peak = fp64_peak_tflops(torch)
        plain["legendre_fp64"] = {}
        for k in ("legendre_alm2map", "legendre_map2alm"):
            lms = pkt["ms"][k] / max(pkt["launches"][k], 1)
            ach = work["legendre_flops"] / (lms / 1e3) / 1e12
            plain["legendre_fp64"][k] = {"ms_per_launch": lms, "achieved_tflops": ach, "peak_tflops": fp64_peak,
                                         "frac": ach / fp64_peak}
        plain["legendre_fp64"]["peak_source"] = "cuBLAS DGEMM 8192^3 measured by bench.py on this GPU"
        head["plain"] = maps_p[:, :4].cpu().numpy()
        head["adjoint"] = {"plain": adjoint_identity(torch, TP, alm, maps_p, T.npix),
                           "split": adjoint_identity(torch, T, alm, maps, T.npix)}
        TP.close()
        del maps_p, alm_p

    for _ in range(a.warmup):
        step(alm)
    torch.cuda.synchronize()

    # ---------------- device-resident timing ----------------
    T.timing(1)
    clocks = ClockSampler(local)
    clocks.start()
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(a.steps):
        step(alm)
    e1.record()
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    kt = T.timing(2)
    T.timing(0)
    ms = 1e3 * reduce_max_seconds(ms / 1e3, dist if world > 1 else None)
    ms_per_step = ms / a.steps
    value = job_rate(world, a.nmaps, a.steps, ms / 1e3)
    head[a.precision] = maps[:, :4].cpu().numpy()  # every step recomputes maps from the same alm

    # ---------------- end to end (host buffers) ----------------
    # every step uploads its alm from pinned host memory and downloads its
    # result; HostPipeline overlaps step i's transform with the upload of
    # i + 1 and the download of i - 1 (copy engines run beside the SMs)
    e2e = None
    if not a.no_e2e:
        from wavemoth_b200.pipeline import HostPipeline
        h_in = torch.from_numpy(alm_h).pin_memory()
        h_out = [torch.empty_like(h_in).pin_memory() for _ in range(2)]

        def e2e_step(d_in, d_out):
            T.alm2map(d_in, out=maps)
            T.map2alm(maps, out=d_out)

        pipe = HostPipeline(alm.shape, alm.dtype, alm.shape, alm.dtype, e2e_step)
        pipe.run([h_in] * 2, h_out)
        torch.cuda.synchronize()

        def e2e_run(n):
            barrier()
            st = torch.cuda.current_stream()
            f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            f0.record(st)
            pipe.run([h_in] * n, [h_out[i & 1] for i in range(n)])
            f1.record(st)
            torch.cuda.synchronize()
            barrier()
            return 1e3 * reduce_max_seconds(f0.elapsed_time(f1) / 1e3, dist if world > 1 else None)

        # the first upload and the last download of a run are not overlapped
        # with a transform; a stream of batches amortises them, so the e2e
        # value is taken over at least --e2e-steps steps (and the K-step figure kept)
        ek = e2e_run(a.steps)
        n_e2e = max(a.steps, a.e2e_steps)
        ems = e2e_run(n_e2e) if n_e2e != a.steps else ek
        nbytes = alm_h.nbytes
        e2e = {"value": job_rate(world, a.nmaps, n_e2e, ems / 1e3), "unit": "maps/s",
               "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes,
               "ms_per_step": ems / n_e2e, "steps": n_e2e,
               "value_at_k_steps": job_rate(world, a.nmaps, a.steps, ek / 1e3),
               "api": "wavemoth_b200.pipeline.HostPipeline over Transform.alm2map/map2alm "
                      "(uploads and downloads overlapped with the neighbouring steps' transforms)"}
        del pipe

    # ---------------- roofline of the dominant kernel ----------------
    kms = {k: (kt["ms"][k] / kt["launches"][k] if kt["launches"][k] else 0.0) for k in kt["ms"]}
    share = {k: kt["ms"][k] / max(sum(kt["ms"].values()), 1e-12) for k in kt["ms"]}
    dominant = max(kt["ms"], key=lambda k: kt["ms"][k])
    peak_hbm, hbm_src = measured_peaks()
    if dominant.startswith("legendre"):
        fp64 = fp64_peak_tflops(torch)
        fp64_achieved = work["legendre_flops"] / (kms[dominant] / 1e3) / 1e12
        fp64_view = {"achieved": fp64_achieved, "peak": fp64, "unit": "TFLOP/s", "frac": fp64_achieved / fp64,
                     "peak_source": "cuBLAS DGEMM 8192^3 measured by bench.py on this GPU",
                     "what": "algorithmic FP64 flops of the transform (2 per multiply-add of 64 vectors, "
                             "5 per recurrence step) over the phase time"}
        if a.precision == "split":
            ops = work["split_int8_ops_" + ("alm2map" if dominant.endswith("alm2map") else "map2alm")]
            achieved = ops / (kms[dominant] / 1e3) / 1e12
            peak = int8_peak_tops(torch)
            src = "cuBLASLt int8 GEMM 8192^3 (torch._int_mm) measured by bench.py on this GPU"
            if peak is None:
                peak, src = 2.0 * measured_peaks_bf16(), "2 x MEASURED_PEAKS.json dense bf16 (int8 rate)"
            roofline = {"bound": "tensor", "kernel": dominant + " (split: residual + level int8 GEMMs)",
                        "achieved": achieved, "peak": peak, "unit": "TOP/s (int8)", "frac": achieved / peak,
                        "peak_source": src, "traffic": profile_traffic(dominant),
                        "int8_ops_per_launch": ops, "fp64_equivalent": fp64_view}
        else:
            roofline = {"bound": "tensor", "kernel": dominant + " (FP64 DMMA)", "achieved": fp64_achieved,
                        "peak": fp64, "unit": "TFLOP/s (fp64)", "frac": fp64_achieved / fp64,
                        "peak_source": fp64_view["peak_source"], "traffic": profile_traffic(dominant),
                        "algorithmic_flops_per_launch": work["legendre_flops"]}
        roofline["hbm_view"] = {"achieved_gbs": (work["matrix_bytes"] + work["legendre_vector_bytes"])
                                / (kms[dominant] / 1e3) / 1e9, "peak_gbs": peak_hbm, "peak_source": hbm_src}
    else:
        achieved = work["ring_bytes"] / (kms[dominant] / 1e3) / 1e9
        roofline = {"bound": "hbm", "kernel": dominant, "achieved": achieved, "peak": peak_hbm,
                    "unit": "GB/s", "frac": achieved / peak_hbm, "peak_source": hbm_src,
                    "traffic": profile_traffic(dominant),
                    "algorithmic_bytes_per_launch": work["ring_bytes"]}
    roofline["kernel_ms_per_launch"] = kms
    roofline["kernel_time_share"] = share
    # the ring kernels against FP64 as well: measured with every global load
    # and store of a ring kernel removed they keep ~80% of their time, so
    # their bound is arithmetic (FFT passes, folds), not HBM
    from wavemoth_b200.healpix import get_ring_pixel_counts
    n = get_ring_pixel_counts(a.nside).astype(np.float64)
    ring_flops = float(np.sum(2.5 * n * np.log2(n))) * a.nmaps
    fp64_ring_peak = fp64_peak_tflops(torch)
    roofline["ring_fp64_view"] = {
        k: {"achieved_tflops": ring_flops / (kms[k] / 1e3) / 1e12, "peak_tflops": fp64_ring_peak,
            "frac": ring_flops / (kms[k] / 1e3) / 1e12 / fp64_ring_peak,
            "hbm_frac": work["ring_bytes"] / (kms[k] / 1e3) / 1e9 / peak_hbm}
        for k in ("ring_synthesis", "ring_analysis")}
    roofline["ring_fp64_view"]["flops_per_launch"] = ring_flops
    roofline["ring_fp64_view"]["what"] = ("nominal real-FFT flops, 2.5 n log2 n per ring of n pixels per map, "
                                          "over the kernel time; peak cuBLAS DGEMM 8192^3 on this GPU")

    # ---------------- parity and CPU baseline (rank 0, N = 1) ----------------
    # maps 0-3 of the batch (seeds 1000-1003) against the reference's own C
    # alm2map of the same alm on the same plan file; the same runner is then
    # timed as the CPU baseline
    cpu, parity, runner = None, None, None
    if rank == 0 and world == 1 and not (a.no_cpu_baseline and a.no_parity):
        try:
            runner = ReferenceRunner(a, path, all_cores=not a.no_cpu_baseline)
        except Exception as ex:  # reported, never fatal for the GPU number
            err = str(ex)[:200]
            parity = {"unavailable": "reference C library: " + err}
            cpu = {"value": None, "unit": "maps/s", "error": err}
    if runner is not None and not a.no_parity:
        parity = headline_parity(runner, head, a.nmaps)
    if runner is not None and not a.no_cpu_baseline:
        try:
            cpu = reference_rate(a, path, a.cpu_baseline_seconds, runner=runner)
        except Exception as ex:
            cpu = {"value": None, "unit": "maps/s", "error": str(ex)[:200]}
        try:
            cpu["map2alm_restatement"] = map2alm_restatement_rate(a, path, a.cpu_baseline_seconds)
        except Exception as ex:
            cpu["map2alm_restatement"] = {"error": str(ex)[:200]}
    elif runner is not None:
        runner.close()
    if parity is not None and "adjoint" in head:
        parity["adjoint_identity"] = head["adjoint"]

    launches = kt["kernels"]  # this library's kernels launched in the timed steps
    out = {
        "metric": METRIC, "value": value, "unit": "maps/s", "n_gpus": world,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms_per_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded N(0,1)(l+1)^-1 alm per map)",
        "config": {"workload": "alm2map+map2alm round trip, nside %d, lmax=mmax %d, %d maps per GPU"
                               % (a.nside, a.lmax, a.nmaps),
                   "nside": a.nside, "lmax": a.lmax, "nmaps_per_gpu": a.nmaps,
                   "precision": ("split: residual products as sliced int8 tcgen05 GEMMs (6 slices, "
                                 "products i+j<=6), FP64 recurrence/levels/rings"
                                 if a.precision == "split" else "plain FP64"),
                   "plain_fp64": plain,
                   "parity_vs_reference": parity,
                   "plan": {"eps": a.eps, "chunk": a.chunk, "memop_cost": a.memop,
                            "max_levels": plan_levels(a)},
                   "parallelism": "replicas (maps sharded per GPU)" if world > 1 else "1 GPU",
                   "l2": "inputs larger than L2 (alm %.2f GB, maps %.2f GB per GPU)"
                         % (alm_h.nbytes / 1e9, T.npix * a.nmaps * 8 / 1e9)},
        "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
        "clocks": clk, "plan_work": work,
    }
    if rank == 0:
        print(json.dumps(out), flush=True)
    T.close()
    if world > 1:
        dist.destroy_process_group()


def run_reference(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    path = ensure_plan(a, 0)
    r = ReferenceRunner(a, path)
    for _ in range(a.warmup):
        r.execute()
    times = [r.execute() for _ in range(a.steps)]
    total = sum(times)
    value = r.plans * r.nmaps * len(times) / (2.0 * total)
    cpu = {"value": value, "unit": "maps/s", "cores": r.threads * r.plans, "kind": "reference",
           "sample": r.describe(len(times))}
    r.close()
    out = {"impl": "reference", "metric": METRIC, "value": value, "unit": "maps/s",
           "n_gpus": int(os.environ.get("WORLD_SIZE", "1")), "steps": a.steps, "warmup": a.warmup,
           "ms_per_step": 1e3 * total / len(times),
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic (seeded N(0,1)(l+1)^-1 alm)",
           "config": {"workload": "alm2map+map2alm round trip, nside %d, lmax=mmax %d; each step "
                                  "a sample of %d maps" % (a.nside, a.lmax, r.plans * r.nmaps),
                      "nside": a.nside, "lmax": a.lmax},
           "cpu_baseline": cpu,
           "e2e": {"value": value, "unit": "maps/s", "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def run_uneven(a):
    """Uneven batch: every request its own plan (nside, 1-8 maps; plans of
    one nside share their device image), all alm2map in split precision,
    captured into one graph by
    wavemoth_b200.batch.Batch; timed against calling the same requests one
    after another on one stream.  Device-resident inputs; L2 is flushed
    between timed launches."""
    import types

    import torch
    from wavemoth_b200.batch import Batch
    from wavemoth_b200.sht import Transform

    rng = np.random.default_rng(2024)
    nsides = [int(x) for x in a.uneven_nsides.split(",")]
    reqs, transforms = [], []
    total_maps = 0
    n2048 = 0
    for i in range(a.requests):
        nside = int(rng.choice(nsides))
        while nside >= 2048 and n2048 >= a.max_nside2048 and len(nsides) > 1:
            nside = int(rng.choice([n for n in nsides if n < 2048]))
        n2048 += nside >= 2048
        nmaps = int(rng.integers(1, 9))
        pa = types.SimpleNamespace(nside=nside, lmax=2 * nside, eps=a.eps, chunk=a.chunk, memop=a.memop,
                                   plan_dir=a.plan_dir, max_levels=a.max_levels)
        # nside 2048 regenerates its residual P at every call: held sliced
        # (80 GB) it would leave no room for the other requests' images
        T = Transform(ensure_plan(pa, 0), nside, 2 * nside, nmaps,
                      precision="split-generate" if nside >= 2048 else "split")
        alm = torch.from_numpy(synthetic_alm(2 * nside, nmaps, 1000 * i)).cuda()
        out = torch.empty((T.npix, nmaps), dtype=torch.float64, device="cuda")
        reqs.append((T, "alm2map", alm, out))
        transforms.append(T)
        total_maps += nmaps
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")  # larger than L2

    def timed(fn):
        for _ in range(a.warmup):
            fn()
        torch.cuda.synchronize()
        ms = 0.0
        for _ in range(a.steps):
            flush.add_(1)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            ms += e0.elapsed_time(e1)
        return ms / a.steps

    def sequential():
        for T, _, alm, out in reqs:
            T.alm2map(alm, out=out)

    seq_ms = timed(sequential)
    cache = a.schedule_cache or tempfile.mktemp(prefix="wm_sched_", suffix=".json")
    t0 = time.time()
    B = Batch(reqs, cache=cache)
    tune_s = time.time() - t0
    width, sms, _ = B.schedule()
    clocks = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    clocks.start()
    batch_ms = timed(B.execute)
    clk = clocks.stop()
    for T in transforms:
        T.device_status()
    line = {"metric": "uneven batch alm2map maps/sec (split precision, one graph launch)",
            "value": total_maps / (batch_ms / 1e3), "unit": "maps/s", "n_gpus": 1, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": batch_ms, "higher_is_better": True, "data": "synthetic",
            "config": {"workload": "uneven batch", "requests": a.requests, "nsides": nsides,
                       "lmax": "2 nside", "maps_per_request": "1-8 (seeded)", "total_maps": total_maps,
                       "request_nsides": [T.nside for T in transforms],
                       "request_maps": [T.nmaps for T in transforms],
                       "request_precisions": [T.precision for T in transforms],
                       "plan_max_levels": plan_levels(a),
                       "schedule": {"graph_branches": width, "sms_per_request": sms or "all",
                                    "search_seconds": tune_s,
                                    "transforms_after_coalescing": B.transforms()},
                       "l2": "flushed between timed launches"},
            "clocks": clk,
            "sequential": {"value": total_maps / (seq_ms / 1e3), "unit": "maps/s", "ms_per_step": seq_ms}}
    B.close()
    for T in transforms:
        T.close()
    print(json.dumps(line), flush=True)


def run_compare_dense(a):
    """Dense-recurrence plans against butterfly plans: one round trip of
    a.nmaps maps per step, device-resident inputs, CUDA-event timed."""
    import types

    import torch
    from wavemoth_b200.sht import Transform
    rows = []
    for nside in [int(x) for x in a.dense_nsides.split(",")]:
        lmax = 2 * nside
        pa = types.SimpleNamespace(nside=nside, lmax=lmax, eps=a.eps, chunk=a.chunk, memop=a.memop,
                                   plan_dir=a.plan_dir, max_levels=a.max_levels)
        path = ensure_plan(pa, 0)
        alm = torch.from_numpy(synthetic_alm(lmax, a.nmaps, 1000)).cuda()
        row = {"nside": nside, "lmax": lmax}
        for prec in ("double", "split"):
            for kind in ("butterfly", "dense"):
                T = Transform(None if kind == "dense" else path, nside, lmax, a.nmaps, precision=prec,
                              dense=kind == "dense")
                maps = torch.empty((T.npix, a.nmaps), dtype=torch.float64, device="cuda")
                out = torch.empty_like(alm)
                for _ in range(a.warmup):
                    T.alm2map(alm, out=maps)
                    T.map2alm(maps, out=out)
                torch.cuda.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                for _ in range(a.steps):
                    T.alm2map(alm, out=maps)
                    T.map2alm(maps, out=out)
                e1.record()
                torch.cuda.synchronize()
                T.device_status()
                row["%s_%s_maps_per_s" % (kind, prec)] = a.nmaps * a.steps / (e0.elapsed_time(e1) / 1e3)
                T.close()
        rows.append(row)
        log(json.dumps(row))
    print(json.dumps({"metric": "alm2map+map2alm maps/sec, dense-recurrence vs butterfly plans",
                      "unit": "maps/s", "nmaps": a.nmaps, "steps": a.steps, "rows": rows}), flush=True)


def main():
    a = parse()
    if a.impl == "reference":
        run_reference(a)
    elif a.compare_dense:
        run_compare_dense(a)
    elif a.uneven:
        run_uneven(a)
    else:
        run_b200(a)


if __name__ == "__main__":
    main()
