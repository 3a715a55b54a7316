"""ctypes drivers of the kernel-level hooks (the reference's
wavemoth/lib.pyx:221-290 and butterfly.pyx:134-161 call patterns), usable on
this library and on the reference's own C library alike."""
import ctypes
import struct

import numpy as np

_dp = ctypes.POINTER(ctypes.c_double)
_sz = ctypes.c_size_t
PULL_FUNC = ctypes.CFUNCTYPE(None, _dp, _sz, _sz, _sz, ctypes.c_void_p, _sz, ctypes.c_void_p)


def dp(a):
    return a.ctypes.data_as(_dp)


def declare_hooks(L):
    L.wavemoth_legendre_transform_auxdata.argtypes = [_sz, _sz, _sz, _dp]
    L.wavemoth_legendre_transform_auxdata.restype = None
    L.wavemoth_legendre_transform.argtypes = [_sz, _sz, _sz] + [_dp] * 6
    L.wavemoth_legendre_transform.restype = None
    L.wavemoth_legendre_transform_sse.argtypes = [_sz, _sz, _sz] + [_dp] * 6 + [ctypes.c_void_p]
    L.wavemoth_legendre_transform_sse.restype = None
    L.wavemoth_legendre_transform_sse_query_work.argtypes = [_sz]
    L.wavemoth_legendre_transform_sse_query_work.restype = _sz
    L.wavemoth_legendre_transform_pack.argtypes = [_sz, _sz, _dp, _dp]
    L.wavemoth_legendre_transform_pack.restype = None
    L.bfm_create_plan.argtypes = [_sz, _sz, _sz, ctypes.c_void_p, ctypes.c_void_p]
    L.bfm_create_plan.restype = ctypes.c_void_p
    L.bfm_destroy_plan.argtypes = [ctypes.c_void_p]
    L.bfm_destroy_plan.restype = None
    L.bfm_transpose_apply_d.argtypes = [ctypes.c_void_p, ctypes.c_void_p, PULL_FUNC, _dp, _sz,
                                        ctypes.c_void_p]
    L.bfm_transpose_apply_d.restype = ctypes.c_int
    L.bfm_scatter.argtypes = [ctypes.c_void_p, _dp, _dp, _dp, _sz, _sz, _sz, ctypes.c_int, ctypes.c_int]
    L.bfm_scatter.restype = ctypes.c_void_p
    return L


def auxdata(L, m, lmin, nk):
    out = np.zeros(max(3 * (nk - 2), 1))
    L.wavemoth_legendre_transform_auxdata(m, lmin, nk, dp(out))
    return out[:3 * max(nk - 2, 0)]


def pack(L, abig, nk):
    nvecs = abig.shape[1]
    out = np.full((nk, nvecs), np.nan)
    L.wavemoth_legendre_transform_pack(nk, nvecs, dp(abig), dp(out))
    return out


def legendre_transform(L, a, x_squared, P0, P1, aux, use_sse=False):
    """lib.pyx:221-279: a is (nk, nvecs); copied into every other row of a
    buffer twice as tall (or packed, for the SSE entry point)."""
    nk, nvecs = a.shape
    nx = x_squared.shape[0]
    abig = np.zeros((2 * nk, nvecs))
    abig[0::2] = a
    y = np.zeros((nx, nvecs))
    aux = np.ascontiguousarray(aux) if aux.size else np.zeros(1)
    args = [dp(np.ascontiguousarray(x_squared)), dp(aux), dp(np.ascontiguousarray(P0)),
            dp(np.ascontiguousarray(P1))]
    if use_sse:
        abuf = pack(L, abig, nk)
        work = np.zeros(max(int(L.wavemoth_legendre_transform_sse_query_work(nvecs)), 16), np.int8)
        L.wavemoth_legendre_transform_sse(nx, nk, nvecs, dp(abuf), dp(y), *args, work.ctypes.data)
    else:
        L.wavemoth_legendre_transform(nx, nk, nvecs, dp(abig), dp(y), *args)
    return y


def transpose_apply(L, matrix_bytes, x):
    """bfm_transpose_apply_d on a serialized matrix with dense residual
    payloads (row_start, row_stop, then a k x n column-major block), the
    pull of DenseResidualButterfly (butterfly.pyx:144-161)."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    nvecs = x.shape[1]
    raw = np.zeros(len(matrix_bytes) + 32, np.uint8)
    off = (-raw.ctypes.data) % 16
    buf = raw[off:off + len(matrix_bytes)]
    buf[:] = np.frombuffer(matrix_bytes, np.uint8)
    nrows, ncols, k_max, nblocks_max = struct.unpack_from("<iiii", matrix_bytes, 0)
    plan = L.bfm_create_plan(max(k_max, nrows, 1), max(nblocks_max, 1), nvecs, None, None)
    out = np.zeros((ncols, nvecs))

    def pull(bufp, start, stop, nv, payload, plen, ctx):
        n = stop - start
        if not n:
            return
        dst = np.ctypeslib.as_array(bufp, shape=(n * nv,)).reshape(n, nv)
        p = payload + ((-payload) % 16)
        rs, re = struct.unpack("<qq", ctypes.string_at(p, 16))
        k = re - rs
        A = np.frombuffer(ctypes.string_at(p + 16, 8 * k * n), np.float64).reshape((k, n), order="F")
        dst[:] = A.T @ x[rs:re]

    cb = PULL_FUNC(pull)
    rc = L.bfm_transpose_apply_d(plan, buf.ctypes.data, cb, dp(out), out.size, None)
    L.bfm_destroy_plan(plan)
    if rc != 0:
        raise RuntimeError("bfm_transpose_apply_d: %d" % rc)
    return out


def scatter(L, mask, t1, t2, src, group, should_add):
    mask = np.ascontiguousarray(mask, dtype=np.int8)
    nvecs = src.shape[1]
    end = L.bfm_scatter(mask.ctypes.data, dp(t1), dp(t2), dp(np.ascontiguousarray(src)),
                        t1.shape[0], t2.shape[0], nvecs, group, should_add)
    return end - mask.ctypes.data
