"""HEALPix ring quadrature weights for the analysis direction.

map2alm with weights computes a_lm = 4 pi / Npix sum_p w_r(p) f_p
lambda_lm(theta_p) e^{-i m phi_p}.  The sum over the pixels of one ring is
an exact quadrature in phi for |m| < n_r / 2, so what is left to correct is
the sum over rings in theta.  The weights here make the quadrature exact for
the zonal harmonics Y_l0, l even, l <= lmax_w (odd l vanish by the north /
south symmetry of the rings): with the 2 Nside ring pairs r (pair 0 the
equator) of n_r pixels per ring and theta_r of the northern ring,

    4 pi / Npix  sum_r c_r n_r w_r lambda_l0(theta_r) = sqrt(4 pi) [l == 0],

c_0 = 1, c_r = 2.  Of the weights satisfying these (fewer equations than
ring pairs), the one closest to all ones in the Euclidean norm is taken
(w = 1 + d, d the least-norm solution of A d = b - A 1).  The lambda_l0 are
this library's FP64 Legendre values (the ylmgen recurrence).  These weights
are this library's construction; the reference has no analysis direction.
"""
import numpy as np

from . import _native
from .healpix import get_ring_pixel_counts, get_ring_thetas, npix


def quadrature_matrix(nside, lmax_w):
    """A[i, r] = 4 pi / Npix c_r n_r lambda_{l,0}(theta_r) for l = 2 i <= lmax_w."""
    thetas = get_ring_thetas(nside, positive_only=True)
    counts = get_ring_pixel_counts(nside)[2 * nside - 1:][:2 * nside]  # equator outwards
    c = np.full(2 * nside, 2.0)
    c[0] = 1.0
    lam = _native.legendre_matrix(0, thetas, lmax_w, epsilon=1e-300)  # (rings, l)
    return (4 * np.pi / npix(nside)) * (c * counts)[None, :] * lam[:, 0:lmax_w + 1:2].T


def ring_weights(nside, lmax_w=None):
    """Weights of the 2 Nside ring pairs (equator first); lmax_w defaults to
    2 Nside."""
    if lmax_w is None:
        lmax_w = 2 * nside
    A = quadrature_matrix(nside, lmax_w)
    b = np.zeros(A.shape[0])
    b[0] = np.sqrt(4 * np.pi)
    one = np.ones(A.shape[1])
    d, *_ = np.linalg.lstsq(A, b - A @ one, rcond=None)
    w = one + d
    if not np.all(w > 0):
        raise ValueError("ring weights not positive for nside %d, lmax_w %d" % (nside, lmax_w))
    return w
