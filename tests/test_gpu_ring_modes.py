"""Ring kernels with both hemispheres of a ring pair in one CTA (default) and
one after the other (the layout of transforms longer than 4096 points,
nside 2048, forced here at small sizes through the test hook
wavemoth_plan_set_hemisphere_mode): synthesis does the same arithmetic per
hemisphere (bitwise equal maps); analysis adds the hemispheres' folds in
one expression or as a read-modify-write of q~ (equal to rounding); both
agree with the oracle."""
import numpy as np
import pytest

from oracle import sht as osht

from .plans import plan_file

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nside,lmax,chunk,nmaps", [(8, 16, 8, 3), (32, 64, 16, 5), (64, 128, 64, 1)])
def test_one_hemisphere_at_a_time_matches(nside, lmax, chunk, nmaps):
    import torch
    from wavemoth_b200 import _native
    from wavemoth_b200.sht import Transform
    path = plan_file(nside, lmax, chunk, 1e-10, 20.0)
    alm = torch.from_numpy(osht.random_alm(lmax, nmaps, seed=91)).cuda()
    maps = torch.from_numpy(np.random.default_rng(92).standard_normal((12 * nside * nside, nmaps))).cuda()
    T = Transform(path, nside, lmax, nmaps)
    m0, a0 = T.alm2map(alm).clone(), T.map2alm(maps).clone()
    assert _native.lib().wavemoth_plan_set_hemisphere_mode(T.plan_handle, 1) == 0
    m1, a1 = T.alm2map(alm).clone(), T.map2alm(maps).clone()
    assert _native.lib().wavemoth_plan_set_hemisphere_mode(T.plan_handle, 0) == 0
    m2 = T.alm2map(alm)
    assert torch.equal(m0, m1) and torch.equal(m0, m2)
    assert float((a0 - a1).abs().max()) <= 1e-13 * float(a0.abs().max())
    want = osht.alm2map_butterfly(osht.Rev1File(path), alm.cpu().numpy(), lmax)
    got = m1.cpu().numpy()
    assert np.linalg.norm(got - want) <= 1e-10 * np.linalg.norm(want)
    T.close()
