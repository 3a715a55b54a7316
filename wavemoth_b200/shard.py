"""One transform over several GPUs: m-sharded Legendre, ring-sharded FFTs,
one all-to-all of q between them.

Every process (one per GPU) holds a ShardedTransform for its part of the
process group.  Part p owns a contiguous range M_p of m (the Legendre
step: ranges balanced by the butterfly matrices' estimated work) and a
contiguous range R_p of ring pairs (the ring FFTs: balanced by pixels):

  alm2map   Legendre of M_p over all rings -> q_leg [ring][m in M_p][parity]
            all-to-all: the block of part k is q_leg's rings R_k (contiguous)
            -> q_x [part k][ring in R_p][m in M_k][parity]
            ring synthesis of R_p -> the pixels of R_p
  map2alm   the reverse: ring analysis of R_p -> q_x [part k][ring in R_p][m in M_k]
            all-to-all -> q_leg [ring][m in M_p], Legendre of M_p -> alm rows of M_p

The exchange is torch.distributed.all_to_all_single: NCCL on CUDA tensors;
with a CPU backend (gloo, used by tests of the multi-process path) the
blocks are staged through host memory.  Layouts are the reference's (alm
complex128 (nalm, nmaps) m-major, maps float64 (npix, nmaps) RING order);
each part holds full-size buffers of which it writes its own rows
(owned_alm_rows, owned_pixel_ranges); gather_map / gather_alm assemble them.
"""
import os

import numpy as np
import torch
import torch.distributed as dist

from . import _native
from .healpix import get_ring_offsets
from .lib import (PRECISION_FLAGS, WAVEMOTH_DENSE, WAVEMOTH_DEVICE_POINTERS, WavemothError, last_error)


def split_sizes(m_bounds, ring_bounds, part, nvecs):
    """Elements (doubles) of every block of the all-to-all, for part `part`:
    alm2map sends q_leg's block for part k (rings R_k, m in M_part) and
    receives part k's block (rings R_part, m in M_k); map2alm the reverse."""
    cnt = np.diff(m_bounds)
    nr = np.diff(ring_bounds)
    send = [int(nr[k] * 2 * cnt[part] * nvecs) for k in range(len(cnt))]
    recv = [int(nr[part] * 2 * cnt[k] * nvecs) for k in range(len(cnt))]
    return send, recv


def owned_pixel_ranges(nside, r0, r1):
    """Pixel ranges of the rings of ring pairs r0 .. r1 - 1 (pair 0 the
    equator): the northern block and the southern one (one range when the
    equator is included)."""
    offs = get_ring_offsets(nside)
    mid = 2 * nside - 1
    north = (int(offs[mid - r1 + 1]), int(offs[mid - r0 + 1]))
    south = (int(offs[mid + r0]), int(offs[mid + r1]))
    if r0 == 0:
        return [(north[0], south[1])]
    return [north, south]


def alm_row(m, lmax):
    """First alm row of m in the m-major layout."""
    return m * (2 * lmax - m + 3) // 2


class ShardedTransform:
    def __init__(self, resource_file, nside, lmax, nmaps=1, group=None, precision="double", dense=False):
        if not torch.cuda.is_available():
            raise RuntimeError("ShardedTransform needs a CUDA device")
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        if self.world < 2:
            raise ValueError("a sharded transform needs at least two processes")
        self.nside, self.lmax, self.nmaps = nside, lmax, nmaps
        self.npix = 12 * nside * nside
        self.nalm = (lmax + 1) * (lmax + 2) // 2
        self.nvecs = 2 * nmaps
        flags = WAVEMOTH_DEVICE_POINTERS | PRECISION_FLAGS[precision] | (WAVEMOTH_DENSE if dense else 0)
        lib = _native.lib()
        p = lib.wavemoth_plan_shard(nside, lmax, lmax, nmaps, flags,
                                    os.fsencode(resource_file) if resource_file else None, self.world, self.rank)
        if not p:
            raise WavemothError("shard plan creation failed: " + last_error())
        self._plan = p
        mb = np.zeros(self.world + 1, np.int64)
        rb = np.zeros(self.world + 1, np.int64)
        if lib.wavemoth_shard_layout(p, mb.ctypes.data, rb.ctypes.data) != 0:
            raise WavemothError("shard layout: " + last_error())
        self.m_bounds, self.ring_bounds = mb, rb
        self.send_a2m, self.recv_a2m = split_sizes(mb, rb, self.rank, self.nvecs)
        dev = torch.device("cuda", torch.cuda.current_device())
        self.q_leg = torch.empty(sum(self.send_a2m), dtype=torch.float64, device=dev)
        self.q_x = torch.empty(sum(self.recv_a2m), dtype=torch.float64, device=dev)
        self.q_ring = torch.empty_like(self.q_x)
        self._nccl = dist.get_backend(group) == "nccl"

    def _stream(self):
        return torch.cuda.current_stream().cuda_stream

    def _check(self, rc, what):
        if rc != 0:
            raise WavemothError("%s failed (%d): %s" % (what, rc, last_error()))

    def _all_to_all(self, out, inp, out_splits, in_splits):
        if self._nccl:
            dist.all_to_all_single(out, inp, out_splits, in_splits, group=self.group)
            return
        torch.cuda.current_stream().synchronize()
        host = torch.empty(out.shape, dtype=out.dtype)
        dist.all_to_all_single(host, inp.cpu(), out_splits, in_splits, group=self.group)
        out.copy_(host)

    def alm2map(self, alm, out=None):
        """Writes the pixels of this part's rings of `out` (npix, nmaps) from
        the full alm (only this part's m rows are read)."""
        if out is None:
            out = torch.zeros((self.npix, self.nmaps), dtype=torch.float64, device=alm.device)
        lib = _native.lib()
        self._check(lib.wavemoth_shard_alm2map_legendre(self._plan, alm.data_ptr(), self.q_leg.data_ptr(),
                                                        self._stream()), "shard alm2map Legendre")
        self._all_to_all(self.q_x, self.q_leg, self.recv_a2m, self.send_a2m)
        self._check(lib.wavemoth_shard_alm2map_rings(self._plan, self.q_x.data_ptr(), self.q_ring.data_ptr(),
                                                     out.data_ptr(), self._stream()), "shard alm2map rings")
        return out

    def map2alm(self, maps, out=None):
        """Writes this part's m rows of `out` (nalm, nmaps) from the full map
        (only this part's rings are read)."""
        if out is None:
            out = torch.zeros((self.nalm, self.nmaps), dtype=torch.complex128, device=maps.device)
        lib = _native.lib()
        self._check(lib.wavemoth_shard_map2alm_rings(self._plan, maps.data_ptr(), self.q_ring.data_ptr(),
                                                     self.q_x.data_ptr(), self._stream()), "shard map2alm rings")
        self._all_to_all(self.q_leg, self.q_x, self.send_a2m, self.recv_a2m)
        self._check(lib.wavemoth_shard_map2alm_legendre(self._plan, self.q_leg.data_ptr(), out.data_ptr(),
                                                        self._stream()), "shard map2alm Legendre")
        return out

    def owned_alm_rows(self, part=None):
        part = self.rank if part is None else part
        return alm_row(int(self.m_bounds[part]), self.lmax), alm_row(int(self.m_bounds[part + 1]), self.lmax)

    def owned_pixel_ranges(self, part=None):
        part = self.rank if part is None else part
        return owned_pixel_ranges(self.nside, int(self.ring_bounds[part]), int(self.ring_bounds[part + 1]))

    def gather_map(self, maps):
        """The full map on every part: each contributes its own pixels."""
        full = torch.zeros_like(maps)
        for a, b in self.owned_pixel_ranges():
            full[a:b] = maps[a:b]
        self._all_reduce(full)
        return full

    def gather_alm(self, alm):
        full = torch.zeros_like(alm)
        a, b = self.owned_alm_rows()
        full[a:b] = alm[a:b]
        self._all_reduce(full)
        return full

    def _all_reduce(self, t):
        if self._nccl:
            dist.all_reduce(t, group=self.group)
            return
        torch.cuda.current_stream().synchronize()
        host = t.cpu()
        dist.all_reduce(host, group=self.group)
        t.copy_(host)

    def close(self):
        if getattr(self, "_plan", None):
            _native.lib().wavemoth_destroy_plan(self._plan)
        self._plan = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
