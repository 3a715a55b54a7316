"""Failure detection without a GPU fault (the reference aborts the process
on any failed check, src/wavemoth_error.h:1-19; this library reports).

* Allocation failure: under a device memory cap plan creation returns NULL
  with the cap named in wavemoth_last_error, and a plan made after the cap
  is lifted works.
* Expired bounded wait: the streamed split-precision GEMM's waits for
  another warp role are cut to one poll through a test hook, so they give
  up; the kernel records a timeout in the plan's device status word, drains
  the copies and MMAs it issued, frees its tensor memory and returns.
  wavemoth_plan_device_status reports WAVEMOTH_ERR_DEVICE once (and clears
  it), and the same plan then computes the right answer with the default
  limit: the context stayed usable.
"""
import ctypes

import numpy as np
import pytest

from oracle import sht as osht
from wavemoth_b200 import _native
from wavemoth_b200.lib import WavemothError

from .plans import plan_file

pytestmark = pytest.mark.gpu

WAVEMOTH_ERR_DEVICE = 4


def test_memory_cap_refuses_plan_then_recovers():
    torch = pytest.importorskip("torch")
    from wavemoth_b200.sht import Transform
    nside, lmax = 16, 32
    path = plan_file(nside, lmax, 8, 1e-10, 1e-10)
    L = _native.lib()
    L.wavemoth_set_device_memory_cap(1024)
    try:
        with pytest.raises(WavemothError, match="cap"):
            Transform(path, nside, lmax, 2)
    finally:
        L.wavemoth_set_device_memory_cap(0)
    alm = osht.random_alm(lmax, 2, seed=5)
    T = Transform(path, nside, lmax, 2)
    got = T.alm2map(torch.from_numpy(alm).cuda()).cpu().numpy()
    T.close()
    want = osht.alm2map_butterfly(osht.Rev1File(path), alm, lmax)
    assert np.linalg.norm(got - want) <= 1e-10 * np.linalg.norm(want)


@pytest.mark.parametrize("direction", ["alm2map", "map2alm"])
def test_expired_wait_reports_device_error(direction):
    torch = pytest.importorskip("torch")
    from wavemoth_b200.sht import Transform
    nside, lmax, nmaps = 32, 64, 3
    path = plan_file(nside, lmax, 16, 1e-10, 20.0)
    L = _native.lib()
    T = Transform(path, nside, lmax, nmaps, precision="split")
    P = Transform(path, nside, lmax, nmaps, precision="double")
    alm = torch.from_numpy(osht.random_alm(lmax, nmaps, seed=9)).cuda()
    src = alm if direction == "alm2map" else P.alm2map(alm)
    run = (lambda t: t.alm2map(src)) if direction == "alm2map" else (lambda t: t.map2alm(src))
    want = run(P)
    torch.cuda.synchronize()

    assert L.wavemoth_plan_set_wait_limit(T._plan, 1) == 0
    run(T)
    rc = L.wavemoth_plan_device_status(T._plan, ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == WAVEMOTH_ERR_DEVICE
    assert "wait" in _native.lib().wavemoth_last_error().decode()
    # the status word is cleared by the read
    assert L.wavemoth_plan_device_status(T._plan, ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)) == 0

    assert L.wavemoth_plan_set_wait_limit(T._plan, 0) == 0
    got = run(T)
    torch.cuda.synchronize()
    T.device_status()
    err = float((got - want).abs().max() / want.abs().max())
    assert err < 1e-9
    T.close()
    P.close()
