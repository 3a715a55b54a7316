"""The N > 1 host logic of bench.py on CPU with gloo (world size 2): every
rank gets its own seeded batch of maps, runs the transform on it (here the
oracle's round trip on a tiny plan), and the job throughput is the maps of
all ranks over the slowest rank's time."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as tmp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, path, out_dir):
    import torch
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    from oracle import sht as osht
    nside, lmax, nmaps = 4, 8, 2
    alm = bench.synthetic_alm(lmax, nmaps, bench.rank_seed(rank, nmaps))
    f = osht.Rev1File(path)
    back = osht.map2alm_butterfly(f, osht.alm2map_butterfly(f, alm, lmax), lmax)
    t = 0.1 * (rank + 1)
    tmax = bench.reduce_max_seconds(t, dist, device="cpu")
    checks = [None] * world
    dist.all_gather_object(checks, float(np.abs(alm).sum()))
    np.save(os.path.join(out_dir, "r%d.npy" % rank),
            np.array([tmax, bench.job_rate(world, nmaps, 1, tmax), checks[0], checks[1],
                      float(np.abs(back).sum())]))
    dist.destroy_process_group()


def test_two_rank_gloo(tmp_path):
    from .plans import plan_file
    path = plan_file(4, 8, 4, 1e-10, 1.0)
    port = _free_port()
    tmp.spawn(_worker, args=(2, port, path, str(tmp_path)), nprocs=2, join=True)
    r0, r1 = np.load(tmp_path / "r0.npy"), np.load(tmp_path / "r1.npy")
    assert r0[0] == pytest.approx(0.2) and r1[0] == pytest.approx(0.2)   # max over ranks
    assert r0[1] == pytest.approx(2 * 2 / 0.2)                          # whole-job maps/s
    assert r0[2] != r0[3]                                               # distinct batches
    assert r0[4] > 0 and r1[4] > 0
