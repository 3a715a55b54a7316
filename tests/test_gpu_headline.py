"""Parity at the headline size: nside 1024, lmax = mmax = 2048, on the plan
file the benchmark uses (ID eps 1e-10, chunk 64, memop cost 20), with the
benchmark's seeded alm (re/im ~ N(0,1)(l+1)^-1, one generator per map).

Tolerances:
  * plain FP64 alm2map against the reference's own C wavemoth_execute
    (oracle/_ref) of the same alm on the same file: <= 1e-10 relative
    (L2 and max-abs over max-abs);
  * split precision alm2map against the same reference output: <= 1e-9
    max-abs over max-abs;
  * map2alm pinned through the adjoint identity
    <alm2map(a), f> = npix / 4 pi <a, map2alm(f)>_c (c_0 = 1, c_m = 2)
    to 1e-11 of |alm2map(a)| |f| (plain) and 1e-10 (split);
  * split round trip map2alm(alm2map(a)) within 1e-9 (max-abs over max-abs)
    of the plain FP64 one.
"""
import os

import numpy as np
import pytest

from oracle import sht as osht

from .plans import plan_file, rel

pytestmark = pytest.mark.gpu

NSIDE, LMAX, NMAPS = 1024, 2048, 2


def _bench_alm(lmax, nmaps, seed0=1000):
    """bench.py's synthetic_alm: map k from its own generator seeded seed0 + k."""
    ls = np.concatenate([np.arange(m, lmax + 1) for m in range(lmax + 1)])
    ms = np.concatenate([np.full(lmax - m + 1, m) for m in range(lmax + 1)])
    out = np.empty((ls.shape[0], nmaps), np.complex128)
    for k in range(nmaps):
        g = np.random.default_rng(seed0 + k)
        re = g.standard_normal(ls.shape[0])
        im = g.standard_normal(ls.shape[0])
        im[ms == 0] = 0.0
        out[:, k] = (re + 1j * im) / (ls + 1.0)
    return out


def _adjoint_error(torch, T, alm, maps, npix):
    g = torch.Generator(device="cuda")
    g.manual_seed(11)
    f = torch.randn(maps.shape, dtype=torch.float64, device="cuda", generator=g)
    b = T.map2alm(f).cpu().numpy()
    errs = []
    for k in range(maps.shape[1]):
        lhs = float((maps[:, k] * f[:, k]).sum())
        rhs = osht.weighted_alm_dot(alm[:, k:k + 1], b[:, k:k + 1], T.lmax) * npix / (4 * np.pi)
        errs.append(abs(lhs - rhs) / float(maps[:, k].norm() * f[:, k].norm()))
    return max(errs)


def test_headline_nside1024_against_reference():
    torch = pytest.importorskip("torch")
    ref = pytest.importorskip("oracle.ref")
    if not ref.available():
        pytest.skip("reference C library (oracle/_ref) not built")
    from wavemoth_b200.sht import Transform

    workers = min(len(os.sched_getaffinity(0)), 32)
    path = plan_file(NSIDE, LMAX, 64, 1e-10, 20.0, workers=workers)
    npix = 12 * NSIDE * NSIDE
    alm = _bench_alm(LMAX, NMAPS)
    rp = ref.RefPlan(NSIDE, LMAX, NMAPS, path, nthreads=8)
    rp.input[:] = alm
    want = rp.execute().copy()
    rp.close()

    d_alm = torch.from_numpy(alm).cuda()
    P = Transform(path, NSIDE, LMAX, NMAPS, precision="double")
    maps_p = P.alm2map(d_alm)
    back_p = P.map2alm(maps_p)
    torch.cuda.synchronize()
    got_p = maps_p.cpu().numpy()
    assert rel(got_p, want) < 1e-10
    assert np.abs(got_p - want).max() <= 1e-10 * np.abs(want).max()
    assert _adjoint_error(torch, P, alm, maps_p, npix) < 1e-11
    back_p = back_p.cpu().numpy()
    P.close()

    S = Transform(path, NSIDE, LMAX, NMAPS, precision="split")
    maps_s = S.alm2map(d_alm)
    back_s = S.map2alm(maps_s)
    torch.cuda.synchronize()
    S.device_status()
    got_s = maps_s.cpu().numpy()
    assert np.abs(got_s - want).max() <= 1e-9 * np.abs(want).max()
    assert np.abs(back_s.cpu().numpy() - back_p).max() <= 1e-9 * np.abs(back_p).max()
    assert _adjoint_error(torch, S, alm, maps_s, npix) < 1e-10
    S.close()
