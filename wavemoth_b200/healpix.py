"""HEALPix ring geometry (RING ordering).

Mirrors wavemoth/healpix.py:5-40 (ring colatitudes, phi offsets, pixel
counts) and the C grid table of src/wavemoth.c:1199-1232 (phi0 per ring and
ring start offsets).  Rings are numbered 0..4*nside-2 from the north pole;
"ring pairs" are numbered from the equator (pair 0 = equator, pair i couples
the rings mid-i and mid+i, mid = 2*nside-1).
"""
import numpy as np


def get_ring_thetas(nside, positive_only=False):
    """Colatitudes of the rings; with positive_only, the 2*nside rings of the
    northern hemisphere ordered from the equator towards the pole."""
    nrings = 4 * nside - 1 if not positive_only else 2 * nside
    i = np.arange(1, nrings + 1, dtype=np.float64)
    z = np.empty(nrings, np.float64)
    z[:nside] = 1 - i[:nside] ** 2 / (3 * nside ** 2)
    z[nside:2 * nside] = 4.0 / 3.0 - (2 * i[nside:2 * nside]) / (3 * nside)
    if positive_only:
        return np.arccos(z[::-1])
    z[2 * nside:] = -z[2 * nside - 2::-1]
    return np.arccos(z)


def get_ring_pixel_counts(nside):
    north = np.arange(4, 4 * nside, 4)
    belt = np.full(2 * nside + 1, 4 * nside, dtype=np.int64)
    south = np.arange(4 * nside - 4, 0, -4)
    return np.concatenate([north, belt, south]).astype(np.int64)


def get_ring_phi0(nside):
    """phi of the first pixel of every ring (src/wavemoth.c:1216-1227)."""
    nrings = 4 * nside - 1
    phi0 = np.empty(nrings)
    for r in range(nrings):
        if r <= nside - 1:
            phi0[r] = np.pi / (4.0 * (r + 1))
        elif r > 3 * nside - 1:
            phi0[r] = np.pi / (4.0 * (nrings - r))
        else:
            phi0[r] = (np.pi / (4.0 * nside)) * (r % 2)
    return phi0


def get_ring_offsets(nside):
    counts = get_ring_pixel_counts(nside)
    return np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)


def npix(nside):
    return 12 * nside * nside


def nalm(lmax, mmax=None):
    mmax = lmax if mmax is None else mmax
    return sum(lmax - m + 1 for m in range(mmax + 1))


def lm_to_idx_mmajor(l, m, lmax):
    """Row of (l, m) in the m-major alm layout (src/wavemoth.c:1017)."""
    return m * (2 * lmax - m + 3) // 2 + (l - m)
