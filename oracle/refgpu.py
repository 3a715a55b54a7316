"""ORACLE (test infrastructure only): the reference's own GPU Legendre kernel
all_transpose_legendre_transforms (wavemoth/cuda/legendre_transform.cu.in:
643-679), built by ``make -C oracle refgpu`` into
oracle/_ref/libwavemoth_ref_gpu_<max rings>.so, and its input format.

``resource(nside, lmax)`` restates the reference's GPU precompute
(wavemoth/cuda/sht.py:98-148 precompute_to_stream, with get_edge :20-35):

    int64 nnz[2 (lmax + 1)]          per (m, odd)
    double x_squared[ni]             cos^2 of the northern rings, equator first
    double Lambda_0[2 (lmax + 1)][ni]   lambda at the first nonzero row of ring i
    double Lambda_1[2 (lmax + 1)][ni]   ... and the row after it
    uint16 i_stops[...]              per m: the even rows' stops, then the odd
                                     rows' (first ring whose lambda is zero)

with the Legendre values of the reference's own ylmgen (oracle/_ref, via
oracle.ref.legendre) at epsilon 1e-30 (sht.py:57).  The kernel computes, per
(m, odd), a[l] = sum_i Lambda_{l}(x_i) q[m, odd, :, i] for one map (2
vectors) with q laid out (lmax + 1, 2, 2, ni).
"""
import ctypes
import os

import numpy as np

from . import ref as _ref

_HERE = os.path.dirname(os.path.abspath(__file__))
_libs = {}


def available(ni):
    return os.path.exists(os.path.join(_HERE, "_ref", "libwavemoth_ref_gpu_%d.so" % ni))


def lib(ni):
    if ni not in _libs:
        L = ctypes.CDLL(os.path.join(_HERE, "_ref", "libwavemoth_ref_gpu_%d.so" % ni))
        L.refgpu_all_transpose.argtypes = [ctypes.c_uint] * 4 + [ctypes.c_void_p] * 4
        L.refgpu_all_transpose.restype = ctypes.c_int
        _libs[ni] = L
    return _libs[ni]


def ring_thetas(nside):
    """healpix.get_ring_thetas(nside, positive_only=True) (wavemoth/healpix.py:5-18)."""
    i = np.arange(1, 2 * nside + 1, dtype=np.float64)
    z = np.where(i <= nside, 1 - i ** 2 / (3.0 * nside ** 2), 4.0 / 3.0 - 2 * i / (3.0 * nside))
    return np.arccos(z[::-1])


def get_edge(Lam):
    """cuda/sht.py:20-35: per row k the first ring whose value is zero
    (i_stops), and every ring's value at its first nonzero row and the row
    after (rings i_stops[k - 1] .. i_stops[k] start at row k).  Vectorised;
    the same values as the reference's loop."""
    zero = Lam == 0
    nk, ni = Lam.shape
    i_stops = np.where(zero.any(axis=1), zero.argmax(axis=1), ni).astype(np.uint16)
    if np.any(i_stops[1:] < i_stops[:-1]):
        raise NotImplementedError("i_stops does not behave nicely")
    start = np.searchsorted(i_stops.astype(np.int64), np.arange(ni), side="right")  # first row of ring i
    cols = np.arange(ni)
    ok = start < nk
    L0 = np.zeros(ni)
    L1 = np.zeros(ni)
    L0[ok] = Lam[start[ok], cols[ok]]
    ok1 = start + 1 < nk
    L1[ok1] = Lam[start[ok1] + 1, cols[ok1]]
    return L0, L1, i_stops


def resource(nside, lmax, epsilon=1e-30):
    thetas = ring_thetas(nside)
    ni = thetas.shape[0]
    nnz = np.zeros(2 * (lmax + 1), np.int64)
    L0 = np.zeros((2 * (lmax + 1), ni))
    L1 = np.zeros((2 * (lmax + 1), ni))
    stops = []
    for m in range(lmax + 1):
        Lam = _ref.legendre(m, thetas, lmax, epsilon)  # (ni, lmax - m + 1)
        for odd in (0, 1):
            sub = np.ascontiguousarray(Lam[:, odd::2].T)
            a, b, s = get_edge(sub) if sub.shape[0] else (np.zeros(ni), np.zeros(ni), np.zeros(0, np.uint16))
            L0[2 * m + odd] = a
            L1[2 * m + odd] = b
            stops.append(s)
            nnz[2 * m + odd] = int(np.sum(sub != 0))
    parts = [nnz.tobytes(), (np.cos(thetas) ** 2).tobytes(), L0.tobytes(), L1.tobytes(),
             np.concatenate(stops).astype(np.uint16).tobytes()]
    return np.frombuffer(b"".join(parts), np.uint8).copy(), int(nnz.sum())


def all_transpose(ni, lmax, resources_ptr, q_ptr, a_ptr, stream=None):
    rc = lib(ni).refgpu_all_transpose(lmax, 0, lmax, ni, resources_ptr, q_ptr, a_ptr, stream)
    if rc != 0:
        raise RuntimeError("reference GPU kernel launch failed: %d" % rc)
