"""Uneven batches of transforms as one CUDA graph launch
(wavemoth_batch_create / _execute in include/wavemoth_b200.h).

Each request is (transform, direction, input, output): a
`wavemoth_b200.sht.Transform`, "alm2map" or "map2alm", and CUDA tensors in
the transform's layouts.  Requests may differ in nside, lmax, number of maps
and precision; no two may use the same Transform (its buffers would race).
Creation captures the requests, longest first, onto parallel graph
branches; `execute()` is then one graph launch on torch's current stream.

Requests of one direction whose Transforms share a device image (same
plan file, lmax and precision) run as one transform of their summed maps:
the matrices are streamed once for all of them (`transforms()` counts what
the graph runs; the results equal the separate calls').

Schedule autotuning: a schedule is the number of branches and, with more
than one, the SMs each request's persistent Legendre kernels may occupy
(the CTAs walking its (m, parity) tile list).  Every candidate (branches 1,
2, 4, 8; SMs all, 1/2, 1/4 of the GPU) is captured and timed over a few
launches, and the fastest kept.  The choice is cached in a JSON file (the
`cache` argument, else $WAVEMOTH_SCHEDULE_CACHE, else
~/.cache/wavemoth_b200/schedules.json) keyed by the batch signature -- the
sorted (nside, lmax, maps, precision, direction) of the requests and the
GPU -- so that a batch of the same shape is built with its schedule at once.
"""
import ctypes
import json
import os

import torch

from . import _native
from .lib import WavemothError, last_error


def _cache_path(cache):
    if cache:
        return cache
    return os.environ.get("WAVEMOTH_SCHEDULE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "wavemoth_b200", "schedules.json"))


def signature(requests):
    """Key of a batch shape: its requests' sizes, precisions and directions
    (sorted) and the GPU."""
    props = torch.cuda.get_device_properties(torch.cuda.current_device())
    reqs = sorted([T.nside, T.lmax, T.nmaps, T.precision, d] for T, d, _, _ in requests)
    return json.dumps({"gpu": props.name, "sms": props.multi_processor_count, "requests": reqs})


def candidate_schedules(nreq, max_width=8):
    sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    out = [(1, 0)]
    w = 2
    while w <= min(nreq, max_width):
        out += [(w, 0), (w, sms // 2), (w, sms // 4)]
        w *= 2
    return out


class Batch:
    def __init__(self, requests, max_width=8, cache=None, retune=False):
        if not requests:
            raise ValueError("empty batch")
        seen = set()
        plans, dirs, ins, outs = [], [], [], []
        self._keep = []
        for T, direction, inp, out in requests:
            if id(T) in seen:
                raise ValueError("two requests share one Transform")
            seen.add(id(T))
            if direction == "alm2map":
                inp, out = T._check_alm(inp), T._check_map(out)
            elif direction == "map2alm":
                inp, out = T._check_map(inp), T._check_alm(out)
            else:
                raise ValueError("direction must be 'alm2map' or 'map2alm'")
            self._keep += [inp, out]
            plans.append(T.plan_handle)
            dirs.append(0 if direction == "alm2map" else 1)
            ins.append(inp.data_ptr())
            outs.append(out.data_ptr())
        n = len(requests)
        vp = ctypes.c_void_p
        self._plans = (vp * n)(*plans)
        self._dirs = (ctypes.c_int * n)(*dirs)
        self._ins = (vp * n)(*ins)
        self._outs = (vp * n)(*outs)
        self._transforms = [r[0] for r in requests]
        stream = torch.cuda.current_stream().cuda_stream
        path = _cache_path(cache)
        key = signature(requests)
        table = {}
        if os.path.exists(path):
            try:
                with open(path) as f:
                    table = json.load(f)
            except (OSError, ValueError):
                table = {}
        cached = None if retune else table.get(key)
        sched = [tuple(cached["schedule"])] if cached else candidate_schedules(n, max_width)
        flat = (ctypes.c_int * (2 * len(sched)))(*[v for pair in sched for v in pair])
        self._batch = _native.lib().wavemoth_batch_create_scheduled(n, self._plans, self._dirs, self._ins, self._outs,
                                                                    flat, len(sched), stream)
        if not self._batch:
            raise WavemothError("batch creation failed: " + last_error())
        self.from_cache = cached is not None
        if not cached:
            width, sms, ms = self.schedule()
            table[key] = {"schedule": [width, sms], "ms": ms}
            try:
                os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
                tmp = path + ".tmp%d" % os.getpid()
                with open(tmp, "w") as f:
                    json.dump(table, f, indent=1, sort_keys=True)
                os.replace(tmp, path)
            except OSError:
                pass  # an unwritable cache only costs the search next time

    def execute(self):
        rc = _native.lib().wavemoth_batch_execute(self._batch, torch.cuda.current_stream().cuda_stream)
        if rc != 0:
            raise WavemothError("batch execute failed (%d): %s" % (rc, last_error()))

    def schedule(self):
        """(graph branches, SMs per request (0: all), measured ms per launch;
        0 when the schedule came from the cache)."""
        w, sms, ms = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
        _native.lib().wavemoth_batch_schedule(self._batch, ctypes.byref(w), ctypes.byref(sms), ctypes.byref(ms))
        return w.value, sms.value, ms.value

    def transforms(self):
        """Transforms the graph runs: requests of one direction on one device
        image are coalesced into one transform of their summed map count."""
        n = _native.lib().wavemoth_batch_transforms(self._batch)
        if n < 0:
            raise WavemothError("batch transforms: " + last_error())
        return n

    def info(self):
        """(number of parallel graph branches chosen, measured ms per launch)."""
        w, ms = ctypes.c_int(), ctypes.c_double()
        _native.lib().wavemoth_batch_info(self._batch, ctypes.byref(w), ctypes.byref(ms))
        return w.value, ms.value

    def close(self):
        if getattr(self, "_batch", None):
            _native.lib().wavemoth_batch_destroy(self._batch)
        self._batch = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
