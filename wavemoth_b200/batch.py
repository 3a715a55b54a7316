"""Uneven batches of transforms as one CUDA graph launch
(wavemoth_batch_create / _execute in include/wavemoth_b200.h).

Each request is (transform, direction, input, output): a
`wavemoth_b200.sht.Transform`, "alm2map" or "map2alm", and CUDA tensors in
the transform's layouts.  Requests may differ in nside, lmax, number of maps
and precision; no two may use the same Transform (its buffers would race).
Creation captures the requests, longest first, onto an autotuned number of
parallel graph branches (it runs every request a few times while timing);
`execute()` is then one graph launch on torch's current stream.
"""
import ctypes

import torch

from . import _native
from .lib import WavemothError, last_error


class Batch:
    def __init__(self, requests, max_width=8):
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
        self._batch = _native.lib().wavemoth_batch_create(n, self._plans, self._dirs, self._ins, self._outs,
                                                          int(max_width), stream)
        if not self._batch:
            raise WavemothError("batch creation failed: " + last_error())

    def execute(self):
        rc = _native.lib().wavemoth_batch_execute(self._batch, torch.cuda.current_stream().cuda_stream)
        if rc != 0:
            raise WavemothError("batch execute failed (%d): %s" % (rc, last_error()))

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
