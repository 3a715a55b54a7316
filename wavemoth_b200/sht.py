"""Torch-facing transforms on device memory.

``Transform`` owns one device-pointer plan per direction over a rev1
resource file and runs alm2map / map2alm on CUDA tensors on torch's current
stream (no host round trip).  Layouts are the reference's: alm complex128
(nalm, nmaps) m-major, maps float64 (12 nside^2, nmaps) RING order.
"""
import os

import torch

from . import _native
from .lib import WAVEMOTH_DEVICE_POINTERS, WAVEMOTH_MMAJOR, WavemothError, last_error


class Transform:
    def __init__(self, resource_file, nside, lmax, nmaps=1, directions=("alm2map", "map2alm")):
        if not torch.cuda.is_available():
            raise RuntimeError("wavemoth_b200.Transform needs a CUDA device")
        self.nside, self.lmax, self.nmaps = nside, lmax, nmaps
        self.npix = 12 * nside * nside
        self.nalm = (lmax + 1) * (lmax + 2) // 2
        self.resource_file = resource_file
        lib = _native.lib()
        self._plans = {}
        for d in directions:
            fn = lib.wavemoth_plan_to_healpix if d == "alm2map" else lib.wavemoth_plan_from_healpix
            p = fn(nside, lmax, lmax, nmaps, 1, None, None, WAVEMOTH_MMAJOR,
                   WAVEMOTH_DEVICE_POINTERS, os.fsencode(resource_file))
            if not p:
                raise WavemothError("plan creation failed: " + last_error())
            self._plans[d] = p

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

    def map2alm(self, maps, out=None):
        maps = self._check_map(maps)
        if out is None:
            out = torch.empty((self.nalm, self.nmaps), dtype=torch.complex128, device=maps.device)
        rc = _native.lib().wavemoth_execute_map2alm_device(
            self._plans["map2alm"], maps.data_ptr(), out.data_ptr(), self._stream())
        if rc != 0:
            raise WavemothError("map2alm failed (%d): %s" % (rc, last_error()))
        return out

    def close(self):
        for p in self._plans.values():
            _native.lib().wavemoth_destroy_plan(p)
        self._plans = {}

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
