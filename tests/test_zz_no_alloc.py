"""The allocation-free Legendre entry point (wavemoth_legendre_alm2map_noalloc).

Callers that cannot allocate device memory when the transform runs (custom
allocator callbacks, frameworks that own all device memory) use this entry
point: its level buffers live in a static device array inside the library.
This test checks, through the C ABI, that two calls in a row produce the
same Legendre-phase output q as the plan's regular path, and that the
device's free memory is the same before and after the first call made after
plan creation (the static array and the kernel's code are loaded when the
plan is created).  The nside 256 case with 8 maps needs more CTA buffers
than the array holds for the plan's usual grid, so it runs on fewer CTAs.
It sits in a file collected last so that a failure here does not hide any
other test result.
"""
import ctypes

import numpy as np
import pytest

from oracle import sht as osht
from wavemoth_b200 import _native
from wavemoth_b200 import lib as wlib

from .plans import plan_file, rel

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("cfg,nmaps", [((16, 32, 8, 1e-10, 1e-10), 3), ((32, 64, 16, 1e-10, 20.0), 2),
                                       ((256, 512, 64, 1e-10, 20.0), 8)])
def test_noalloc_matches_plan_path(cfg, nmaps):
    torch = pytest.importorskip("torch")
    nside, lmax, chunk, eps, memop = cfg
    path = plan_file(nside, lmax, chunk, eps, memop)
    alm = osht.random_alm(lmax, nmaps, seed=77)
    out = np.zeros((12 * nside * nside, nmaps))
    plan = wlib.ShtPlan(nside, lmax, lmax, alm, out, "mmajor", matrix_data_filename=path)
    plan.perform_legendre_transform()
    want = plan.get_work()

    d_alm = torch.from_numpy(alm.view(np.float64).copy()).cuda()
    nq = 2 * (lmax + 1) * 2 * nside * 2 * nmaps
    L = _native.lib()
    for call in range(2):
        d_q = torch.full((nq,), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        rc = L.wavemoth_legendre_alm2map_noalloc(plan._plan, ctypes.c_void_p(d_alm.data_ptr()),
                                                 ctypes.c_void_p(d_q.data_ptr()), None)
        assert rc == 0, wlib.last_error()
        torch.cuda.synchronize()
        if call == 0:
            assert torch.cuda.mem_get_info()[0] == free0
        got = d_q.cpu().numpy().view(np.complex128).reshape(want.shape)
        assert np.all(np.isfinite(got))
        assert rel(got, want) < 1e-12
    plan.close()
