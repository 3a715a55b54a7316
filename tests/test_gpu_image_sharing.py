"""Plans of one resource file share their device image (program, tables,
sliced P and W): a second plan allocates only its own per-call buffers, keeps
working after the first is destroyed, and computes what a plan of its own
would (bitwise)."""
import numpy as np
import pytest

from oracle import sht as osht

from .plans import plan_file

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["double", "split"])
def test_second_plan_shares_the_image(precision):
    import torch
    from wavemoth_b200.sht import Transform
    nside, lmax = 32, 64
    path = plan_file(nside, lmax, 16, 1e-10, 20.0)
    alm = torch.from_numpy(osht.random_alm(lmax, 3, seed=71)).cuda()
    T1 = Transform(path, nside, lmax, 3, precision=precision)
    want = T1.alm2map(alm).clone()
    w1 = T1.work()
    assert 0 < w1["image_bytes"] < w1["device_bytes"]
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    T2 = Transform(path, nside, lmax, 3, precision=precision)
    torch.cuda.synchronize()
    used = free0 - torch.cuda.mem_get_info()[0]
    w2 = T2.work()
    assert w2["image_bytes"] == w1["image_bytes"]
    own = w2["device_bytes"] - w2["image_bytes"]
    # the driver rounds allocations up; the image is not allocated again
    assert used < own + w1["image_bytes"] // 2 + (8 << 20)
    T1.close()
    got = T2.alm2map(alm)
    T2.device_status()
    assert torch.equal(got, want)
    T2.close()


def test_other_precision_gets_its_own_image():
    from wavemoth_b200.sht import Transform
    nside, lmax = 16, 32
    path = plan_file(nside, lmax, 8, 1e-10, 1e-10)
    Td = Transform(path, nside, lmax, 1, precision="double")
    Ts = Transform(path, nside, lmax, 1, precision="split")
    assert Ts.work()["image_bytes"] > Td.work()["image_bytes"]
    alm = osht.random_alm(lmax, 1, seed=5)
    import torch
    a = torch.from_numpy(alm).cuda()
    md, ms = Td.alm2map(a).cpu().numpy(), Ts.alm2map(a).cpu().numpy()
    assert np.abs(ms - md).max() <= 1e-9 * np.abs(md).max()
    Td.close()
    Ts.close()
