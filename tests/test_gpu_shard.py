"""The m-sharded transform's own kernels under torch.distributed: 2 and 3
processes on this GPU (gloo; the all-to-all staged through host memory, so
no kernel waits on another process), each running its part's Legendre and
ring kernels.  The assembled map and alm equal the single-plan transform's
(1e-13 relative, max-abs over max-abs: the parts run the same kernels on
the same matrices; only the work split differs), both precisions, a
butterfly plan and a dense-recurrence plan."""
import os
import socket
import tempfile

import numpy as np
import pytest

from oracle import sht as osht

from .plans import plan_file

pytestmark = pytest.mark.gpu


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, path, nside, lmax, precision, dense, out):
    import torch
    import torch.distributed as dist
    from wavemoth_b200.shard import ShardedTransform
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        alm = torch.from_numpy(np.load(os.path.join(out, "alm.npy"))).cuda()
        f = torch.from_numpy(np.load(os.path.join(out, "f.npy"))).cuda()
        T = ShardedTransform(None if dense else path, nside, lmax, alm.shape[1], precision=precision, dense=dense)
        maps = T.gather_map(T.alm2map(alm))
        back = T.gather_alm(T.map2alm(f))
        torch.cuda.synchronize()
        if rank == 0:
            np.save(os.path.join(out, "maps.npy"), maps.cpu().numpy())
            np.save(os.path.join(out, "back.npy"), back.cpu().numpy())
        T.close()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,precision,dense", [(2, "double", False), (3, "double", False),
                                                   (2, "split", False), (2, "double", True)])
def test_sharded_transform_matches_single_plan(world, precision, dense):
    torch = pytest.importorskip("torch")
    import torch.multiprocessing as mp
    from wavemoth_b200.sht import Transform
    nside, lmax, nmaps = 32, 64, 3
    path = plan_file(nside, lmax, 16, 1e-10, 20.0)
    out = tempfile.mkdtemp(prefix="wm_shard_")
    alm = osht.random_alm(lmax, nmaps, seed=12)
    f = np.random.default_rng(13).standard_normal((12 * nside * nside, nmaps))
    np.save(os.path.join(out, "alm.npy"), alm)
    np.save(os.path.join(out, "f.npy"), f)
    mp.start_processes(_worker, args=(world, free_port(), path, nside, lmax, precision, dense, out),
                       nprocs=world, start_method="spawn")
    T = Transform(None if dense else path, nside, lmax, nmaps, precision=precision, dense=dense)
    want_map = T.alm2map(torch.from_numpy(alm).cuda()).cpu().numpy()
    want_alm = T.map2alm(torch.from_numpy(f).cuda()).cpu().numpy()
    T.close()
    got_map = np.load(os.path.join(out, "maps.npy"))
    got_alm = np.load(os.path.join(out, "back.npy"))
    assert np.abs(got_map - want_map).max() <= 1e-13 * np.abs(want_map).max()
    assert np.abs(got_alm - want_alm).max() <= 1e-13 * np.abs(want_alm).max()
