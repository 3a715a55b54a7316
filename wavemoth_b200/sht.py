"""Torch-facing transforms on device memory.

``Transform`` owns one device-pointer plan per direction over a rev1
resource file and runs alm2map / map2alm on CUDA tensors on torch's current
stream (no host round trip).  Layouts are the reference's: alm complex128
(nalm, nmaps) m-major, maps float64 (12 nside^2, nmaps) RING order.
"""
import os

import torch

from . import _native
from .lib import (PRECISION_FLAGS, WAVEMOTH_DENSE, WAVEMOTH_DEVICE_POINTERS, WAVEMOTH_MMAJOR, WavemothError,
                  last_error)


class Transform:
    """Both directions share one device plan (the compiled butterfly program
    serves A^T for alm2map and A for map2alm).  precision='split' runs the
    residual and level products as sliced int8 tensor-core GEMMs re-summed in
    FP64 ('split-generate': the residual P regenerated at every call instead
    of held sliced in device memory)."""

    def __init__(self, resource_file, nside, lmax, nmaps=1, precision="double", dense=False):
        """dense=True: no butterfly file (resource_file may be None); every
        (m, parity) block is one three-term recurrence over all rings,
        seeded by the device's FP64 Legendre generator."""
        if not torch.cuda.is_available():
            raise RuntimeError("wavemoth_b200.Transform needs a CUDA device")
        self.nside, self.lmax, self.nmaps = nside, lmax, nmaps
        self.npix = 12 * nside * nside
        self.nalm = (lmax + 1) * (lmax + 2) // 2
        self.resource_file = resource_file
        if precision not in PRECISION_FLAGS:
            raise ValueError("precision must be one of %s" % ", ".join(PRECISION_FLAGS))
        self.precision = precision
        flags = WAVEMOTH_DEVICE_POINTERS | PRECISION_FLAGS[precision] | (WAVEMOTH_DENSE if dense else 0)
        lib = _native.lib()
        p = lib.wavemoth_plan_to_healpix(nside, lmax, lmax, nmaps, 1, None, None, WAVEMOTH_MMAJOR, flags,
                                         os.fsencode(resource_file) if resource_file else None)
        if not p:
            raise WavemothError("plan creation failed: " + last_error())
        self._plan = p
        self._plans = {"alm2map": p, "map2alm": p}

    def _stream(self):
        return torch.cuda.current_stream().cuda_stream

    def _check_alm(self, alm):
        if alm.dtype != torch.complex128 or not alm.is_cuda or tuple(alm.shape) != (self.nalm, self.nmaps):
            raise ValueError("alm must be a CUDA complex128 tensor of shape (%d, %d)"
                             % (self.nalm, self.nmaps))
        return alm.contiguous()

    def _check_map(self, m):
        if m.dtype != torch.float64 or not m.is_cuda or tuple(m.shape) != (self.npix, self.nmaps):
            raise ValueError("map must be a CUDA float64 tensor of shape (%d, %d)"
                             % (self.npix, self.nmaps))
        return m.contiguous()

    def alm2map(self, alm, out=None):
        alm = self._check_alm(alm)
        if out is None:
            out = torch.empty((self.npix, self.nmaps), dtype=torch.float64, device=alm.device)
        rc = _native.lib().wavemoth_execute_alm2map_device(
            self._plans["alm2map"], alm.data_ptr(), out.data_ptr(), self._stream())
        if rc != 0:
            raise WavemothError("alm2map failed (%d): %s" % (rc, last_error()))
        return out

    def map2alm(self, maps, out=None, niter=0):
        """a = 4 pi / Npix A^T f (times the ring weights, if set); niter > 0
        refines it by Jacobi iterations a += map2alm(f - alm2map(a))."""
        maps = self._check_map(maps)
        if out is None:
            out = torch.empty((self.nalm, self.nmaps), dtype=torch.complex128, device=maps.device)
        if niter:
            rc = _native.lib().wavemoth_map2alm_iterative_device(
                self._plans["map2alm"], maps.data_ptr(), out.data_ptr(), int(niter), self._stream())
        else:
            rc = _native.lib().wavemoth_execute_map2alm_device(
                self._plans["map2alm"], maps.data_ptr(), out.data_ptr(), self._stream())
        if rc != 0:
            raise WavemothError("map2alm failed (%d): %s" % (rc, last_error()))
        return out

    def set_ring_weights(self, weights):
        """Quadrature weights of the 2 Nside ring pairs (equator first) used by
        map2alm (wavemoth_b200.weights.ring_weights), or None for unit
        weights."""
        import ctypes

        import numpy as np
        if weights is None:
            rc = _native.lib().wavemoth_plan_set_ring_weights(self._plan, None)
        else:
            w = np.ascontiguousarray(weights, dtype=np.float64)
            if w.shape != (2 * self.nside,):
                raise ValueError("weights must have shape (%d,)" % (2 * self.nside))
            rc = _native.lib().wavemoth_plan_set_ring_weights(
                self._plan, w.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        if rc != 0:
            raise WavemothError("set_ring_weights failed: " + last_error())

    def device_status(self):
        """Waits for torch's current stream and raises if a kernel recorded an
        error in the plan's device status word (e.g. an expired bounded wait)."""
        rc = _native.lib().wavemoth_plan_device_status(self._plan, self._stream())
        if rc != 0:
            raise WavemothError("device status (%d): %s" % (rc, last_error()))

    @property
    def plan_handle(self):
        return self._plan

    def timing(self, mode):
        """Per-kernel event timing: mode 1 enable/reset, 0 disable, 2 read
        -> dict of milliseconds and launch counts."""
        import ctypes
        out = (ctypes.c_double * 8)()
        rc = _native.lib().wavemoth_plan_timing(self._plan, mode, out)
        if rc != 0:
            raise WavemothError("timing failed: " + last_error())
        if mode != 2:
            return None
        keys = ("legendre_alm2map", "legendre_map2alm", "ring_synthesis", "ring_analysis")
        return {"ms": dict(zip(keys, list(out)[:4])), "launches": dict(zip(keys, list(out)[4:])),
                "kernels": int(_native.lib().wavemoth_plan_kernel_launches(self._plan))}

    def work(self):
        """Algorithmic work of one direction (see wavemoth_plan_work)."""
        import ctypes
        out = (ctypes.c_double * 12)()
        rc = _native.lib().wavemoth_plan_work(self._plan, self.nmaps, out)
        if rc != 0:
            raise WavemothError("work query failed: " + last_error())
        o = list(out)
        return {"legendre_flops": o[0], "matrix_bytes": o[1], "legendre_vector_bytes": o[2],
                "ring_bytes": o[3], "interp_elems": o[4], "rec_elems": o[5], "dense_elems": o[6],
                "legendre_grid": o[7],
                "split_elems_alm2map": o[8], "split_elems_map2alm": o[9],
                "split_int8_ops_alm2map": o[10], "split_int8_ops_map2alm": o[11],
                "device_bytes": _native.lib().wavemoth_plan_device_bytes(self._plan),
                "program_bytes": _native.lib().wavemoth_plan_program_bytes(self._plan),
                "image_bytes": _native.lib().wavemoth_plan_image_bytes(self._plan)}

    def close(self):
        if getattr(self, "_plan", None):
            _native.lib().wavemoth_destroy_plan(self._plan)
        self._plan = None
        self._plans = {}

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
