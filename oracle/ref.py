"""ORACLE (test infrastructure only): ctypes access to the reference's own C
library, compiled from the reference's sources by ``make -C oracle ref``
into oracle/_ref/libwavemoth_ref.so (see oracle/Makefile for the shims).

``RefPlan`` mirrors the Cython ShtPlan of wavemoth/lib.pyx:113-193: it binds
an m-major complex alm input and an (npix, nmaps) map output at plan time and
runs the reference's wavemoth_execute / wavemoth_perform_legendre_transforms.
"""
import contextlib
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(_HERE, "_ref", "libwavemoth_ref.so")
_lib = None
MAX_THREADS = 8


def available():
    """The reference library is built, or can be built from the checkout
    named by WAVEMOTH_REFERENCE."""
    ref = os.environ.get("WAVEMOTH_REFERENCE")
    return os.path.exists(REF_LIB) or bool(ref and os.path.isdir(os.path.join(ref, "src")))


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(REF_LIB):
            ref = os.environ.get("WAVEMOTH_REFERENCE")
            if not ref:
                raise RuntimeError("oracle/_ref/libwavemoth_ref.so is not built; run "
                                   "make -C oracle ref REF=<reference checkout> or set "
                                   "WAVEMOTH_REFERENCE")
            subprocess.run(["make", "-C", _HERE, "ref", "REF=" + ref], check=True,
                           capture_output=True)
        L = ctypes.CDLL(REF_LIB)
        dp = ctypes.POINTER(ctypes.c_double)
        L.wavemoth_plan_to_healpix.restype = ctypes.c_void_p
        L.wavemoth_plan_to_healpix.argtypes = [ctypes.c_int] * 5 + [dp, dp, ctypes.c_int,
                                                                    ctypes.c_uint, ctypes.c_char_p]
        for name in ("wavemoth_execute", "wavemoth_destroy_plan",
                     "wavemoth_perform_legendre_transforms", "wavemoth_perform_backward_ffts",
                     "wavemoth_disable_phase_shifting"):
            getattr(L, name).argtypes = [ctypes.c_void_p]
            getattr(L, name).restype = None
        L.wavemoth_get_legendre_flops.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        L.wavemoth_get_legendre_flops.restype = ctypes.c_int64
        L.wavemoth_query_resourcefile.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_int),
                                                  ctypes.POINTER(ctypes.c_int)]
        L.wavemoth_query_resourcefile.restype = ctypes.c_int
        L.refhook_get_work.argtypes = [ctypes.c_void_p, dp]
        L.refhook_get_work.restype = None
        L.refhook_set_ncpus.argtypes = [ctypes.c_int]
        L.refhook_set_ncpus.restype = None
        L.refhook_phi0s.argtypes = [ctypes.c_int, dp]
        L.refhook_phi0s.restype = ctypes.c_int
        L.refhook_legendre.argtypes = [ctypes.c_int, dp, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_double, dp]
        L.refhook_legendre.restype = ctypes.c_int
        L.refhook_worker_sizes_ok.argtypes = [ctypes.c_void_p]
        L.refhook_worker_sizes_ok.restype = ctypes.c_int
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


@contextlib.contextmanager
def stdout_to_stderr():
    """The reference prints progress to stdout while loading a plan
    (src/wavemoth.c:695-699); keep stdout clean for JSON output."""
    import sys
    sys.stdout.flush()
    saved = os.dup(1)
    try:
        os.dup2(2, 1)
        yield
    finally:
        os.dup2(saved, 1)
        os.close(saved)


def legendre(m, thetas, lmax, epsilon=1e-300):
    th = np.ascontiguousarray(thetas, dtype=np.float64)
    out = np.empty((th.shape[0], lmax - m + 1))
    rc = lib().refhook_legendre(int(m), _dp(th), th.shape[0], int(lmax), float(epsilon), _dp(out))
    if rc != 0:
        raise ValueError("refhook_legendre: %d" % rc)
    return out


def phi0s(nside):
    out = np.empty(4 * nside - 1)
    lib().refhook_phi0s(int(nside), _dp(out))
    return out


def query_resourcefile(path):
    n, l = ctypes.c_int(), ctypes.c_int()
    rc = lib().wavemoth_query_resourcefile(path.encode(), ctypes.byref(n), ctypes.byref(l))
    return rc, n.value, l.value


PULL_FUNC = ctypes.CFUNCTYPE(None, ctypes.POINTER(ctypes.c_double), ctypes.c_size_t,
                             ctypes.c_size_t, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_size_t,
                             ctypes.c_void_p)


def bfm_transpose_apply(matrix_bytes, x, mode="rows"):
    """The reference's own bfm_transpose_apply_d (src/butterfly.c.in:375-432)
    on a serialized matrix, with the pull callbacks of its Python test
    harness: mode "rows" copies input rows (ButterflyPlan,
    butterfly.pyx:134-141), mode "dense" applies a dense residual payload
    (DenseResidualButterfly, butterfly.pyx:144-161)."""
    import struct
    L = lib()
    x = np.ascontiguousarray(x, dtype=np.float64)
    nvecs = x.shape[1]
    raw = np.zeros(len(matrix_bytes) + 32, np.uint8)
    off = (-raw.ctypes.data) % 16
    buf = raw[off:off + len(matrix_bytes)]
    buf[:] = np.frombuffer(matrix_bytes, np.uint8)
    nrows, ncols, k_max, nblocks_max = struct.unpack_from("<iiii", matrix_bytes, 0)
    sems = (ctypes.c_char * 64)()
    L.bfm_create_plan.restype = ctypes.c_void_p
    L.bfm_create_plan.argtypes = [ctypes.c_size_t] * 3 + [ctypes.c_void_p] * 2
    L.bfm_transpose_apply_d.restype = ctypes.c_int
    L.bfm_transpose_apply_d.argtypes = [ctypes.c_void_p, ctypes.c_void_p, PULL_FUNC,
                                        ctypes.POINTER(ctypes.c_double), ctypes.c_size_t,
                                        ctypes.c_void_p]
    plan = L.bfm_create_plan(max(k_max, max(nrows, 1)), max(nblocks_max, 1), nvecs,
                             ctypes.addressof(sems), ctypes.addressof(sems) + 32)
    out = np.zeros((ncols, nvecs))

    def pull(bufp, start, stop, nv, payload, plen, ctx):
        n = stop - start
        dst = np.ctypeslib.as_array(bufp, shape=(max(n, 1) * nv,))[:n * nv].reshape(n, nv) if n else None
        if mode == "rows":
            if n:
                dst[:] = x[start:stop]
            return
        p = payload + ((-payload) % 16)
        rs, re = struct.unpack("<qq", ctypes.string_at(p, 16))
        k = re - rs
        if n:
            A = np.frombuffer(ctypes.string_at(p + 16, 8 * k * n), np.float64).reshape((k, n), order="F")
            dst[:] = A.T @ x[rs:re]

    cb = PULL_FUNC(pull)
    rc = L.bfm_transpose_apply_d(plan, buf.ctypes.data, cb,
                                 out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), out.size, None)
    if rc != 0:
        raise RuntimeError("bfm_transpose_apply_d: %d" % rc)
    return out


class RefPlan:
    def __init__(self, nside, lmax, nmaps, resource_file, nthreads=1, phase_shifts=True,
                 attempts=50):
        L = lib()
        self.nside, self.lmax, self.nmaps = nside, lmax, nmaps
        nalm = (lmax + 1) * (lmax + 2) // 2
        self.input = np.zeros((nalm, nmaps), np.complex128)
        self.output = np.zeros((12 * nside * nside, nmaps))
        # one CPU per presented NUMA node, at most 8 nodes (see ref_hooks.c)
        nthreads = max(1, min(int(nthreads), MAX_THREADS, len(os.sched_getaffinity(0))))
        self.nthreads = nthreads
        L.refhook_set_ncpus(nthreads)
        self.plan = None
        for _ in range(attempts):
            with stdout_to_stderr():
                plan = L.wavemoth_plan_to_healpix(nside, lmax, lmax, nmaps, nthreads,
                                                  _dp(self.input.view(np.float64)),
                                                  _dp(self.output), 0, 0,
                                                  resource_file.encode())
            if not plan:
                raise RuntimeError("reference plan creation failed")
            if L.refhook_worker_sizes_ok(plan):
                self.plan = plan
                break
            # a worker lost the unsynchronised size reduction; this plan
            # would trip the reference's own assert, so build it again
            L.wavemoth_destroy_plan(plan)
        if not self.plan:
            raise RuntimeError("reference plan creation kept racing (%d attempts)" % attempts)
        if not phase_shifts:
            L.wavemoth_disable_phase_shifting(self.plan)

    def execute(self):
        lib().wavemoth_execute(self.plan)
        return self.output

    def perform_legendre_transforms(self):
        lib().wavemoth_perform_legendre_transforms(self.plan)

    def get_work(self):
        ni = 2 * self.nside
        out = np.zeros((self.lmax + 1, 2, ni, self.nmaps), np.complex128)
        lib().refhook_get_work(self.plan, _dp(out.view(np.float64)))
        return out

    def legendre_flops(self, m, odd):
        return lib().wavemoth_get_legendre_flops(self.plan, m, odd)

    def close(self):
        if self.plan:
            lib().wavemoth_destroy_plan(self.plan)
            self.plan = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
