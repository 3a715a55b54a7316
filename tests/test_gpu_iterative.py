"""Ring quadrature weights and iterative (Jacobi) map2alm.

The oracle is the butterfly restatement in oracle/sht.py on the same plan
file: weighted map2alm = map2alm of the map with every ring's pixels
multiplied by its weight; the iteration a_{k+1} = a_k +
map2alm(f - alm2map(a_k)) run in numpy with the oracle's alm2map and
map2alm.  Tolerance 1e-10 relative (max-abs over max-abs), the plain path's
bound.  The iteration itself must drive the band-limited round-trip error
down (lmax = nside: each step shrinks it)."""
import numpy as np
import pytest

from oracle import sht as osht
from wavemoth_b200 import weights as wts
from wavemoth_b200.healpix import get_ring_offsets

from .plans import plan_file

pytestmark = pytest.mark.gpu


def weight_map(nside, w):
    """Per-pixel weight: ring pair |r| of every ring."""
    offs = get_ring_offsets(nside)
    mid = 2 * nside - 1
    out = np.empty(12 * nside * nside)
    for ring in range(4 * nside - 1):
        out[offs[ring]:offs[ring + 1]] = w[abs(ring - mid)]
    return out


def maxrel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


@pytest.mark.parametrize("cfg", [(16, 32, 8, 1e-10, 1e-10), (32, 64, 16, 1e-10, 20.0)])
def test_weighted_map2alm_matches_oracle(cfg):
    torch = pytest.importorskip("torch")
    from wavemoth_b200.sht import Transform
    nside, lmax, chunk, eps, memop = cfg
    path = plan_file(nside, lmax, chunk, eps, memop)
    w = wts.ring_weights(nside)
    f = np.random.default_rng(1).standard_normal((12 * nside * nside, 2))
    T = Transform(path, nside, lmax, 2)
    T.set_ring_weights(w)
    got = T.map2alm(torch.from_numpy(f).cuda()).cpu().numpy()
    T.set_ring_weights(None)
    plain = T.map2alm(torch.from_numpy(f).cuda()).cpu().numpy()
    T.close()
    rf = osht.Rev1File(path)
    assert maxrel(got, osht.map2alm_butterfly(rf, f * weight_map(nside, w)[:, None], lmax)) < 1e-10
    assert maxrel(plain, osht.map2alm_butterfly(rf, f, lmax)) < 1e-10


@pytest.mark.parametrize("weighted", [False, True])
def test_iterative_map2alm(weighted):
    torch = pytest.importorskip("torch")
    from wavemoth_b200.sht import Transform
    nside, lmax = 16, 16
    path = plan_file(nside, lmax, 8, 1e-12, 20.0)
    rf = osht.Rev1File(path)
    a_true = osht.random_alm(lmax, 2, seed=4)
    f = osht.alm2map_butterfly(rf, a_true, lmax)
    w = wts.ring_weights(nside) if weighted else None
    wm = weight_map(nside, w)[:, None] if weighted else 1.0
    T = Transform(path, nside, lmax, 2)
    if weighted:
        T.set_ring_weights(w)
    errs = []
    a_ref = osht.map2alm_butterfly(rf, f * wm, lmax)
    for niter in range(4):
        got = T.map2alm(torch.from_numpy(f).cuda(), niter=niter).cpu().numpy()
        if niter:
            a_ref = a_ref + osht.map2alm_butterfly(rf, (f - osht.alm2map_butterfly(rf, a_ref, lmax)) * wm, lmax)
        assert maxrel(got, a_ref) < 1e-10
        errs.append(maxrel(got, a_true))
    T.close()
    assert all(e1 < e0 for e0, e1 in zip(errs, errs[1:])), errs
    assert errs[-1] < 1e-3 * errs[0], errs
