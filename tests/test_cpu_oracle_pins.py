"""Pins of the oracle against the reference and against known answers."""
import numpy as np
import pytest
import scipy.special

from oracle import sht as osht
from wavemoth_b200 import _native, healpix


def ref_or_skip():
    from oracle import ref
    if not ref.available():
        pytest.skip("reference C library not available")
    return ref


@pytest.mark.parametrize("nside,lmax", [(4, 8), (32, 64), (128, 256)])
def test_legendre_bitwise_equal_to_reference_ylmgen(nside, lmax):
    ref = ref_or_skip()
    th = np.concatenate([osht.ring_thetas(nside, positive_only=True), [0.0, np.pi, np.pi / 2, 1e-3]])
    for m in sorted(set(list(range(0, lmax + 1, max(1, lmax // 11))) + [lmax])):
        for eps in (1e-300, 1e-30):
            assert np.array_equal(osht.normalized_legendre(m, th, lmax, eps),
                                  ref.legendre(m, th, lmax, eps))


@pytest.mark.parametrize("theta,m,lmax", [(np.pi / 2, 0, 10), (np.pi / 4, 0, 10),
                                          (3 * np.pi / 4, 0, 10), (np.pi / 4, 1, 4),
                                          (np.pi / 4, 2, 4), (np.pi / 4, 50, 50),
                                          (np.pi / 2, 49, 50), (0.001, 250, 300)])
def test_legendre_normalisation(theta, m, lmax):
    """wavemoth/test/test_legendre.py:9-26 (scipy's sph_harm is now sph_harm_y)."""
    got = osht.normalized_legendre(m, [theta], lmax)[0]
    want = np.real(scipy.special.sph_harm_y(np.arange(m, lmax + 1), m, theta, 0.0))
    np.testing.assert_allclose(got, want, rtol=1e-10, atol=1e-300)


@pytest.mark.parametrize("nside,lmax", [(16, 32), (256, 512)])
def test_product_legendre_matches_oracle(nside, lmax):
    th = osht.ring_thetas(nside, positive_only=True)
    for m in (0, 1, lmax // 3, lmax - 1, lmax):
        a = osht.normalized_legendre(m, th, lmax)
        b = _native.legendre_matrix(m, th, lmax)
        assert np.abs(a - b).max() <= 1e-12 * np.abs(a).max()


def test_recurrence_coefficients_match():
    ref = ref_or_skip()
    import ctypes
    L = ref.lib()
    L.wavemoth_legendre_transform_auxdata.argtypes = [ctypes.c_size_t] * 3 + [ctypes.c_void_p]
    for m, lmin, nk in [(0, 0, 40), (10, 210, 30), (300, 301, 200), (1000, 1000, 500)]:
        want = np.empty(3 * (nk - 2))
        L.wavemoth_legendre_transform_auxdata(m, lmin, nk, want.ctypes.data)
        assert np.array_equal(osht.legendre_auxdata(m, lmin, nk), want)
        np.testing.assert_allclose(_native.recurrence_coefficients(m, lmin, nk), want, rtol=1e-14)


@pytest.mark.parametrize("nvecs", [2, 4, 6, 10])
@pytest.mark.parametrize("nx", [1, 2, 3, 7, 11])
@pytest.mark.parametrize("nk", [2, 3, 6, 11])
def test_recurrence_transform(nvecs, nx, nk):
    """wavemoth/test/test_legendre_transforms.py:22-72: nside 2048, m = 10,
    lmin = m + 200, rings from 340: the strip recurrence equals the dense
    product with ylmgen's Lambda."""
    nside, ixmin, m = 2048, 340, 10
    lmin = m + 200
    lstop = lmin + 2 * nk
    nodes = osht.ring_thetas(nside, positive_only=True)[ixmin:ixmin + nx]
    P = osht.normalized_legendre(m, nodes, lstop, 1e-30).T[(lmin - m):(lstop - m):2, :]
    a = np.arange(nk * nvecs, dtype=np.float64).reshape(nk, nvecs)
    y0 = (a.T @ P).T
    y = osht.legendre_transform(a, np.cos(nodes) ** 2, osht.legendre_auxdata(m, lmin, nk), P[0], P[1])
    np.testing.assert_allclose(y, y0, rtol=1e-12, atol=1e-12 * np.abs(y0).max())


def test_healpix_geometry():
    """wavemoth/test/test_healpix.py:41-71 and test_wavemoth.py:119-121."""
    nside = 4
    th = healpix.get_ring_thetas(nside)
    assert th.shape == (4 * nside - 1,)
    pos = healpix.get_ring_thetas(nside, positive_only=True)
    assert pos[0] == np.arccos(0)
    np.testing.assert_allclose(pos, th[:2 * nside][::-1])
    c = healpix.get_ring_pixel_counts(nside)
    assert len(c) == 4 * nside - 1 and c[0] == 4 and c[-1] == 4
    assert c[2 * nside] == 4 * nside and c.sum() == 12 * nside ** 2 and np.all(c == c[::-1])
    np.testing.assert_array_equal(healpix.get_ring_phi0(16), osht.grid(16)[0])


def test_c_grid_table_matches():
    from wavemoth_b200 import lib
    phi0, offs, mid, npix = lib.get_healpix_grid(16)
    np.testing.assert_array_equal(phi0, osht.grid(16)[0])
    np.testing.assert_array_equal(offs, osht.grid(16)[1])
    assert mid == 31 and npix == 12 * 256
    np.testing.assert_array_equal(lib._get_healpix_phi0s(16), healpix.get_ring_phi0(16))
    ref = pytest.importorskip("oracle.ref")
    if ref.available():
        np.testing.assert_array_equal(ref.phi0s(16), phi0)


def test_ring_weights_integrate_zonal_harmonics():
    """Ring weights (wavemoth_b200.weights): the weighted ring sum integrates
    Y_l0, l even <= 2 nside, exactly (checked against an independent
    Legendre evaluation: numpy's Legendre series, lambda_l0 = sqrt((2l+1)/4pi)
    P_l(cos theta)), and stays close to unit weights."""
    import numpy as np
    from numpy.polynomial import legendre as L
    from wavemoth_b200 import weights
    from wavemoth_b200.healpix import get_ring_pixel_counts, get_ring_thetas
    for nside in (4, 16, 32):
        w = weights.ring_weights(nside)
        th = get_ring_thetas(nside, positive_only=True)
        n = get_ring_pixel_counts(nside)[2 * nside - 1:]
        c = np.where(np.arange(2 * nside) == 0, 1.0, 2.0)
        for l in range(0, 2 * nside + 1, 2):
            coef = np.zeros(l + 1)
            coef[l] = 1.0
            ylm = np.sqrt((2 * l + 1) / (4 * np.pi)) * L.legval(np.cos(th), coef)
            q = 4 * np.pi / (12 * nside * nside) * np.sum(c * n * w * ylm)
            assert abs(q - (np.sqrt(4 * np.pi) if l == 0 else 0.0)) < 1e-12
        assert 0.9 < w.min() and w.max() < 1.15


def test_native_recurrence_last_row_matches_numpy_loop():
    """The plan writer's stability check (wm_host_recurrence_last_row) runs the
    residual recurrence of src/legendre_transform.c.in:680-716 per column."""
    import numpy as np
    from wavemoth_b200 import _native
    rng = np.random.default_rng(3)
    m, lmin, nk, nx = 7, 9, 40, 33
    aux = _native.recurrence_coefficients(m, lmin, nk)
    x2 = rng.uniform(0, 1, nx)
    P0, P1 = rng.standard_normal(nx), rng.standard_normal(nx)
    pp, p = P0.copy(), P1.copy()
    for k in range(2, nk):
        al, be, ga = aux[3 * (k - 2):3 * (k - 2) + 3]
        pp, p = p, (x2 + al) * be * p + ga * pp
    got = _native.recurrence_last_row(x2, P0, P1, aux, nk)
    assert np.allclose(got, p, rtol=1e-12, atol=0)
    assert np.array_equal(_native.recurrence_last_row(x2, P0, P1, aux[:0], 1), P0)
