"""ctypes binding of ``libwavemoth_b200.so`` (the in-tree native library).

The library holds the CUDA kernels, the host plan code and the C-ABI of
include/wavemoth.h and include/wavemoth_b200.h.  Loading fails loudly when it
has not been built: there is no fallback implementation.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libwavemoth_b200.so")

_lib = None

c_double_p = ctypes.POINTER(ctypes.c_double)
c_int_p = ctypes.POINTER(ctypes.c_int)
c_int64_p = ctypes.POINTER(ctypes.c_int64)


class NativeLibraryMissing(RuntimeError):
    pass


# ctypes signatures of the host tools of the plan-file writer
HOST_SIGNATURES = {
    "wm_host_legendre": (ctypes.c_int, [ctypes.c_int, c_double_p, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_double, c_double_p]),
    "wm_host_recurrence_coefficients": (None, [ctypes.c_int64, ctypes.c_int64, ctypes.c_int64,
                                               c_double_p]),
    "wm_host_recurrence_last_row": (None, [c_double_p, c_double_p, c_double_p, c_double_p, ctypes.c_int64,
                                            ctypes.c_int64, c_double_p]),
    "wm_host_interp_decomp": (ctypes.c_int, [c_double_p, ctypes.c_int, ctypes.c_int,
                                             ctypes.c_double, c_int_p, c_int_p, c_double_p]),
}


def _declare(lib):
    sig = HOST_SIGNATURES
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    try:
        from . import _abi
        _abi.declare(lib)
    except ImportError:
        pass


def lib():
    """The loaded native library (raises NativeLibraryMissing if absent)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise NativeLibraryMissing(
                "%s is missing: build it with `python -m wavemoth_b200.build`" % LIB_PATH)
        _lib = ctypes.CDLL(LIB_PATH)
        _declare(_lib)
    return _lib


def dptr(a):
    return a.ctypes.data_as(c_double_p)


def ipt(a):
    return a.ctypes.data_as(c_int_p)


def legendre_matrix(m, thetas, lmax, epsilon=1e-300):
    """(ntheta, lmax-m+1) matrix of normalised lambda_lm(theta); the same
    contract as wavemoth/legendre.pyx:24-57."""
    th = np.ascontiguousarray(thetas, dtype=np.float64)
    out = np.empty((th.shape[0], lmax - m + 1), np.float64)
    rc = lib().wm_host_legendre(int(m), dptr(th), th.shape[0], int(lmax), float(epsilon), dptr(out))
    if rc != 0:
        raise ValueError("wm_host_legendre failed (%d)" % rc)
    return out


def recurrence_coefficients(m, lmin, nk):
    """(alpha, beta, gamma) triples, 3*(nk-2) values (src/legendre_transform.c.in:723-747)."""
    if nk < 3:
        return np.zeros(0)
    out = np.empty(3 * (nk - 2), np.float64)
    lib().wm_host_recurrence_coefficients(int(m), int(lmin), int(nk), dptr(out))
    return out


def recurrence_last_row(x2, P0, P1, aux, nk):
    """Row nk-1 of the three-term recurrence started from (P0, P1), per column."""
    x2, P0, P1 = (np.ascontiguousarray(v, dtype=np.float64) for v in (x2, P0, P1))
    aux = np.ascontiguousarray(aux, dtype=np.float64)
    if aux.size < 3 * max(0, nk - 2):
        raise ValueError("recurrence coefficients too short")
    out = np.empty(x2.shape[0], np.float64)
    lib().wm_host_recurrence_last_row(dptr(x2), dptr(P0), dptr(P1), dptr(aux) if aux.size else None,
                                      x2.shape[0], int(nk), dptr(out))
    return out


def interp_decomp(A, eps):
    """Precision-eps interpolative decomposition of A (rows, cols).

    Returns (krank, perm, proj) with A[:, perm[krank:]] ~= A[:, perm[:krank]] @ proj.
    """
    m, n = A.shape
    buf = np.array(A, dtype=np.float64, order="F", copy=True)
    perm = np.empty(n, np.intc)
    k = ctypes.c_int(0)
    proj = np.empty(max(1, min(m, n) * n), np.float64)
    lib().wm_host_interp_decomp(dptr(buf), m, n, float(eps), ctypes.byref(k), ipt(perm), dptr(proj))
    k = k.value
    proj = proj[:k * (n - k)].reshape((k, n - k), order="F").copy()
    return k, perm.astype(np.int64), proj
