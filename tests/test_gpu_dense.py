"""Dense-recurrence plans (WAVEMOTH_DENSE; no butterfly file): every
(m, parity) block one three-term recurrence over all rings from the first
row with lambda_lm > 1e-30, seeded on the device by the FP64 ylmgen walk.

Tolerances: against the oracle's dense transform (ylmgen values times alm,
exact per-ring DFT) 1e-12 relative L2 -- the dense path has no compression,
only the recurrence's rounding; against the reference C library on an
ID-eps 1e-10 butterfly file 1e-9 (that file's compression error); split
precision on a dense plan within 1e-9 (max-abs over max-abs) of the FP64
dense path; map2alm pinned to the oracle's dense adjoint at 1e-12."""
import numpy as np
import pytest

from oracle import sht as osht

from .plans import plan_file, rel

pytestmark = pytest.mark.gpu

CASES = [(8, 16), (16, 32), (32, 64), (64, 128)]


@pytest.mark.parametrize("nside,lmax", CASES)
def test_dense_alm2map_map2alm_against_oracle(nside, lmax):
    torch = pytest.importorskip("torch")
    from wavemoth_b200.sht import Transform
    alm = osht.random_alm(lmax, 3, seed=nside)
    T = Transform(None, nside, lmax, 3, dense=True)
    maps = T.alm2map(torch.from_numpy(alm).cuda())
    f = np.random.default_rng(2).standard_normal((12 * nside * nside, 3))
    back = T.map2alm(torch.from_numpy(f).cuda())
    torch.cuda.synchronize()
    T.close()
    assert rel(maps.cpu().numpy(), osht.alm2map_dense(nside, alm, lmax)) < 1e-12
    assert rel(back.cpu().numpy(), osht.map2alm_dense(nside, f, lmax)) < 1e-12


def test_dense_against_reference_c_library():
    torch = pytest.importorskip("torch")
    ref = pytest.importorskip("oracle.ref")
    if not ref.available():
        pytest.skip("reference C library not built")
    from wavemoth_b200.sht import Transform
    nside, lmax = 64, 128
    path = plan_file(nside, lmax, 64, 1e-10, 20.0)
    alm = osht.random_alm(lmax, 1, seed=2024)
    rp = ref.RefPlan(nside, lmax, 1, path, nthreads=4)
    rp.input[:] = alm
    want = rp.execute().copy()
    rp.close()
    T = Transform(None, nside, lmax, 1, dense=True)
    got = T.alm2map(torch.from_numpy(alm).cuda()).cpu().numpy()
    T.close()
    assert rel(got, want) < 1e-9


@pytest.mark.parametrize("nside,lmax", [(16, 32), (64, 128)])
def test_dense_split_precision(nside, lmax):
    torch = pytest.importorskip("torch")
    from wavemoth_b200.sht import Transform
    alm = torch.from_numpy(osht.random_alm(lmax, 5, seed=9)).cuda()
    P = Transform(None, nside, lmax, 5, dense=True)
    S = Transform(None, nside, lmax, 5, dense=True, precision="split")
    mp, ms = P.alm2map(alm), S.alm2map(alm)
    ap, as_ = P.map2alm(mp), S.map2alm(mp)
    torch.cuda.synchronize()
    S.device_status()
    assert float((ms - mp).abs().max()) <= 1e-9 * float(mp.abs().max())
    assert float((as_ - ap).abs().max()) <= 1e-9 * float(ap.abs().max())
    P.close()
    S.close()
