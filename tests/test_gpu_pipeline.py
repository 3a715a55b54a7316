"""HostPipeline: streamed host batches give the same results as direct calls."""
import numpy as np
import pytest
import torch

from oracle import sht as osht

from .plans import plan_file

pytestmark = pytest.mark.gpu


def test_pipeline_round_trip_matches_direct_calls():
    from wavemoth_b200.pipeline import HostPipeline
    from wavemoth_b200.sht import Transform
    nside, lmax, nmaps = 16, 32, 3
    T = Transform(plan_file(nside, lmax, 8, 1e-10, 20.0), nside, lmax, nmaps)
    maps = torch.empty((T.npix, nmaps), dtype=torch.float64, device="cuda")

    def step(d_in, d_out):
        T.alm2map(d_in, out=maps)
        T.map2alm(maps, out=d_out)

    ins = [torch.from_numpy(osht.random_alm(lmax, nmaps, seed=70 + i)).pin_memory() for i in range(5)]
    outs = [torch.empty_like(x).pin_memory() for x in ins]
    pipe = HostPipeline(ins[0].shape, ins[0].dtype, ins[0].shape, ins[0].dtype, step)
    pipe.run(ins, outs)
    torch.cuda.synchronize()
    for x, y in zip(ins, outs):
        want = T.map2alm(T.alm2map(x.cuda())).cpu()
        assert torch.equal(y, want)
    T.close()
