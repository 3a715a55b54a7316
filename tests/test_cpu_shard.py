"""Host logic of the m-sharded transform (wavemoth_b200.shard), no GPU:

* the all-to-all block sizes agree between senders and receivers and cover
  the Legendre-side and ring-side buffers exactly;
* two gloo ranks exchange Legendre-side q blocks (values encoding ring, m,
  parity and vector) with all_to_all_single at those sizes, and the
  exchange-table addressing of the ring-side gather kernel (restated here
  as the kernel computes it: row pair of m at tab[2m] + ring tab[2m + 1])
  finds every value where the ring kernel expects it; the reverse
  direction likewise;
* the parts' pixel ranges cover every pixel once.
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from wavemoth_b200.shard import owned_pixel_ranges, split_sizes


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def layout(nparts, mmax, ni):
    mb = np.linspace(0, mmax + 1, nparts + 1).round().astype(np.int64)
    rb = np.linspace(0, ni, nparts + 1).round().astype(np.int64)
    return mb, rb


def exchange_table(mb, rb, part, mmax, nvecs):
    """The table the plan uploads (abi.cpp, shard exchange table)."""
    tab = np.zeros(2 * (mmax + 1), np.int64)
    r0, r1 = rb[part], rb[part + 1]
    seg = 0
    for s in range(len(mb) - 1):
        m0, cnt = mb[s], mb[s + 1] - mb[s]
        for m in range(m0, m0 + cnt):
            tab[2 * m] = seg + (m - m0) * 2 * nvecs
            tab[2 * m + 1] = cnt * 2 * nvecs
        seg += (r1 - r0) * cnt * 2 * nvecs
    return tab


def code(ring, m, par, v):
    return ring * 1e6 + m * 1e2 + par * 10 + v


def _worker(rank, world, port, mmax, ni, nvecs, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mb, rb = layout(world, mmax, ni)
        send, recv = split_sizes(mb, rb, rank, nvecs)
        m0, m1 = mb[rank], mb[rank + 1]
        # alm2map: Legendre side [ring][m in M_rank][parity][v]
        leg = np.array([code(r, m, p, v) for r in range(ni) for m in range(m0, m1) for p in range(2)
                        for v in range(nvecs)], np.float64)
        x = torch.empty(sum(recv), dtype=torch.float64)
        dist.all_to_all_single(x, torch.from_numpy(leg), recv, send)
        x = x.numpy()
        tab = exchange_table(mb, rb, rank, mmax, nvecs)
        r0, r1 = rb[rank], rb[rank + 1]
        ok = True
        for rl in range(r1 - r0):
            for m in range(mmax + 1):
                base = tab[2 * m] + rl * tab[2 * m + 1]
                for p in range(2):
                    for v in range(nvecs):
                        ok &= x[base + p * nvecs + v] == code(r0 + rl, m, p, v)
        # map2alm: ring side scattered into [part k][ring in R_rank][m in M_k], exchanged back
        ring_side = np.array([code(r0 + rl, m, p, v) for rl in range(r1 - r0) for m in range(mmax + 1)
                              for p in range(2) for v in range(nvecs)], np.float64)
        xs = np.empty(sum(recv))
        for rl in range(r1 - r0):
            for m in range(mmax + 1):
                base = tab[2 * m] + rl * tab[2 * m + 1]
                xs[base:base + 2 * nvecs] = ring_side[(rl * (mmax + 1) + m) * 2 * nvecs:][:2 * nvecs]
        back = torch.empty(sum(send), dtype=torch.float64)
        dist.all_to_all_single(back, torch.from_numpy(xs), send, recv)
        ok &= bool(np.array_equal(back.numpy(), leg))
        q.put((rank, bool(ok)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_exchange_layout_two_processes(world):
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    mp.start_processes(_worker, args=(world, free_port(), 9, 6, 4, q), nprocs=world, start_method="spawn")
    res = dict(q.get() for _ in range(world))
    assert all(res[r] for r in range(world)), res


def test_split_sizes_consistent():
    mb, rb = layout(4, 20, 16)
    nvecs = 6
    sends = [split_sizes(mb, rb, p, nvecs)[0] for p in range(4)]
    recvs = [split_sizes(mb, rb, p, nvecs)[1] for p in range(4)]
    for a in range(4):
        for b in range(4):
            assert sends[a][b] == recvs[b][a]
        assert sum(sends[a]) == 16 * 2 * (mb[a + 1] - mb[a]) * nvecs
        assert sum(recvs[a]) == (rb[a + 1] - rb[a]) * 2 * 21 * nvecs


@pytest.mark.parametrize("nside", [1, 2, 8, 16])
def test_pixel_ranges_cover_once(nside):
    ni = 2 * nside
    for nparts in (2, 3):
        if nparts > ni:
            continue
        _, rb = layout(nparts, 0, ni)
        seen = np.zeros(12 * nside * nside, np.int64)
        for p in range(nparts):
            for a, b in owned_pixel_ranges(nside, int(rb[p]), int(rb[p + 1])):
                seen[a:b] += 1
        assert np.all(seen == 1)
