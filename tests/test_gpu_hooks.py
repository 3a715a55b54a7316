"""Kernel-level hooks that compute on the GPU, against the reference's own
C library (oracle/_ref) and the exact products:

* wavemoth_legendre_transform{,_sse}: the sweep of
  wavemoth/test/test_legendre_transforms.py:22-72 (Nside 2048, rings
  340 .. 340 + nx, m = 10, lmin = 210, nx and nk small, 2..22 vectors, the
  auxdata read at offset 0 or 1 of a buffer), y against P^T a to 7 decimals
  (the reference test's assert_almost_equal) and the plain entry point bit
  for bit against the reference's scalar routine;
* bfm_transpose_apply_d: wavemoth/test/test_butterfly.py:370-389 (A = i j,
  20 x 10, chunk 3, dense residual payloads, 1, 2 and 200 levels) against
  A^T x (rtol 1e-12) and the reference's apply;
* wavemoth_execute_adjoint: against the other direction's plan scaled by
  npix / 4 pi (alm2map plan) resp. 4 pi / npix (map2alm plan), 1e-12.
"""
import io

import numpy as np
import pytest

from oracle import sht as osht
from wavemoth_b200 import _native
from wavemoth_b200 import lib as wlib
from wavemoth_b200.healpix import get_ring_thetas
from wavemoth_b200.resource import ArrayProvider, butterfly_compress, serialize_butterfly_matrix

from . import hooks_util as H
from .plans import plan_file

pytestmark = pytest.mark.gpu

NSIDE, IXMIN, M = 2048, 340, 10


def _ref():
    from oracle import ref
    if not ref.available():
        pytest.skip("reference C library not available")
    return H.declare_hooks(ref.lib())


def _case(nvecs, nx, nk):
    lmin = M + 200
    lstop = lmin + 2 * nk
    nodes = get_ring_thetas(NSIDE, positive_only=True)[IXMIN:IXMIN + nx]
    P = _native.legendre_matrix(M, nodes, lstop, epsilon=1e-30)
    P = np.ascontiguousarray(P.T[(lmin - M):(lstop - M):2, :])
    x_squared = np.cos(nodes) ** 2
    a = np.arange(nk * nvecs, dtype=np.float64).reshape(nk, nvecs)
    return lmin, P, x_squared, a


@pytest.mark.parametrize("nvecs", [2, 4, 6, 10, 12, 22])
@pytest.mark.parametrize("nk", [2, 3, 4, 6, 7, 10, 11, 62, 64, 66])
@pytest.mark.parametrize("nx", [1, 2, 3, 4, 6, 7, 10, 11])
def test_legendre_transform_sweep(nvecs, nx, nk):
    ours = H.declare_hooks(_native.lib())
    lmin, P, x_squared, a = _case(nvecs, nx, nk)
    y0 = (a.T @ P).T
    for auxalign in (0, 1):
        buf = np.zeros(max(3 * (nk - 2), 0) + auxalign)
        buf[auxalign:] = H.auxdata(ours, M, lmin, nk)
        aux = buf[auxalign:]
        for use_sse in (False, True):
            y = H.legendre_transform(ours, a, x_squared, P[0], P[1], aux, use_sse=use_sse)
            np.testing.assert_almost_equal(y, y0, decimal=7)


@pytest.mark.parametrize("nvecs", [2, 6, 22])
@pytest.mark.parametrize("nk", [2, 7, 66])
def test_legendre_transform_bitwise_reference(nvecs, nk):
    ours, ref = H.declare_hooks(_native.lib()), _ref()
    lmin, P, x_squared, a = _case(nvecs, 11, nk)
    aux = H.auxdata(ours, M, lmin, nk)
    y = H.legendre_transform(ours, a, x_squared, P[0], P[1], aux)
    y_ref = H.legendre_transform(ref, a, x_squared, P[0], P[1], aux)
    assert np.array_equal(y, y_ref)


@pytest.mark.parametrize("num_levels", [1, 2, 200])
def test_bfm_transpose_apply_dense_residual(num_levels):
    ours = H.declare_hooks(_native.lib())
    i, j = np.ogrid[:20, :10]
    A = (i * j).astype(np.float64)
    tree = butterfly_compress(A, chunk_size=3)
    stream = io.BytesIO()
    stream.write(b"a" * 160)
    data = serialize_butterfly_matrix(tree, ArrayProvider(A), stream=stream,
                                      num_levels=num_levels).getvalue()[160:]
    x = np.arange(40, dtype=np.float64).reshape(20, 2)
    y = H.transpose_apply(ours, data, x)
    np.testing.assert_allclose(y, A.T @ x, rtol=1e-12, atol=1e-9)
    from oracle import ref
    if ref.available():
        np.testing.assert_allclose(y, ref.bfm_transpose_apply(data, x, mode="dense"), rtol=1e-13, atol=1e-10)


@pytest.mark.parametrize("chunk", [1, 3, 5, 9])
def test_bfm_transpose_apply_roundtrip(chunk):
    """test_butterfly.py:294-313 through this library: A^T I recovers A."""
    ours = H.declare_hooks(_native.lib())
    A = np.arange(1, 101, dtype=np.float64).reshape(10, 10)
    data = serialize_butterfly_matrix(butterfly_compress(A, chunk), ArrayProvider(A)).getvalue()
    At = H.transpose_apply(ours, data, np.eye(10))
    np.testing.assert_allclose(At.T, A, rtol=1e-9, atol=1e-9)


@pytest.mark.parametrize("cfg", [(8, 16, 8, 1e-10, 1.0), (32, 64, 16, 1e-10, 20.0)])
def test_execute_adjoint(cfg):
    nside, lmax, chunk, eps, memop = cfg
    path = plan_file(nside, lmax, chunk, eps, memop)
    npix, nmaps = 12 * nside * nside, 3
    rng = np.random.default_rng(5)
    f = rng.standard_normal((npix, nmaps))
    alm = np.zeros(((lmax + 1) * (lmax + 2) // 2, nmaps), np.complex128)
    p = wlib.ShtPlan(nside, lmax, lmax, alm, f.copy(), "mmajor", matrix_data_filename=path)
    got = p.execute_adjoint().copy()
    p.close()
    q = wlib.ShtPlan(nside, lmax, lmax, np.ascontiguousarray(f), np.zeros_like(alm), "mmajor",
                     matrix_data_filename=path, direction="map2alm")
    want = q.execute().copy() * (npix / (4 * np.pi))
    q.close()
    assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()
    # the map2alm plan's adjoint is (4 pi / npix) alm2map
    a = osht.random_alm(lmax, nmaps, seed=8)
    r = wlib.ShtPlan(nside, lmax, lmax, np.zeros((npix, nmaps)), np.ascontiguousarray(a), "mmajor",
                     matrix_data_filename=path, direction="map2alm")
    got_m = r.execute_adjoint().copy()
    r.close()
    s = wlib.ShtPlan(nside, lmax, lmax, np.ascontiguousarray(a), np.zeros((npix, nmaps)), "mmajor",
                     matrix_data_filename=path)
    want_m = s.execute().copy() * (4 * np.pi / npix)
    s.close()
    assert np.abs(got_m - want_m).max() <= 1e-12 * np.abs(want_m).max()
