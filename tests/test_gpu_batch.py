"""Uneven batches in one graph launch (wavemoth_b200.batch): requests of
different nside, lmax = 2 nside, 1..8 maps, both directions and both
precisions.  Each request's output must equal (bitwise) the output of the
same transform called alone, on two launches in a row; the split-precision
requests are also checked against the oracle's butterfly transform at the
split tolerance (max |error| <= 1e-9 max |value|).
"""
import numpy as np
import pytest
import torch

from oracle import sht as osht

from .plans import plan_file

pytestmark = pytest.mark.gpu


def _transform(nside, nmaps, precision):
    from wavemoth_b200.sht import Transform
    lmax = 2 * nside
    return Transform(plan_file(nside, lmax, 16, 1e-10, 20.0), nside, lmax, nmaps, precision=precision)


def test_uneven_batch_matches_single_calls():
    from wavemoth_b200.batch import Batch
    rng = np.random.default_rng(55)
    specs = [(nside, int(rng.integers(1, 9)), prec, direction)
             for nside, prec, direction in [(8, "split", "alm2map"), (16, "double", "alm2map"),
                                            (32, "split", "alm2map"), (16, "split", "map2alm"),
                                            (8, "double", "map2alm"), (32, "double", "alm2map"),
                                            (64, "split", "alm2map")]]
    reqs, singles, alms = [], [], []
    for i, (nside, nmaps, prec, direction) in enumerate(specs):
        T = _transform(nside, nmaps, prec)
        if direction == "alm2map":
            a = osht.random_alm(T.lmax, nmaps, seed=600 + i)
            inp = torch.from_numpy(a).cuda()
            out = torch.empty((T.npix, nmaps), dtype=torch.float64, device="cuda")
            single = T.alm2map(inp).clone()
        else:
            a = rng.standard_normal((T.npix, nmaps))
            inp = torch.from_numpy(a).cuda()
            out = torch.empty((T.nalm, nmaps), dtype=torch.complex128, device="cuda")
            single = T.map2alm(inp).clone()
        alms.append(a)
        reqs.append((T, direction, inp, out))
        singles.append(single)
    import tempfile
    cache = tempfile.mktemp(prefix="wm_sched_", suffix=".json")
    B = Batch(reqs, cache=cache)
    width, ms = B.info()
    assert width in (1, 2, 4, 8) and ms > 0 and not B.from_cache
    # a batch of the same shape takes the cached schedule without a search
    B2 = Batch(reqs, cache=cache)
    assert B2.from_cache and B2.schedule()[:2] == B.schedule()[:2]
    B2.close()
    for _ in range(2):
        for r in reqs:
            r[3].zero_()
        B.execute()
        torch.cuda.synchronize()
        for r, s in zip(reqs, singles):
            assert torch.equal(r[3], s)
    for (nside, nmaps, prec, direction), (T, _, _, out), a in zip(specs, reqs, alms):
        T.device_status()
        if prec == "split" and direction == "alm2map":
            path = plan_file(nside, 2 * nside, 16, 1e-10, 20.0)
            want = osht.alm2map_butterfly(osht.Rev1File(path), a, 2 * nside)
            got = out.cpu().numpy()
            assert np.abs(got - want).max() <= 1e-9 * np.abs(want).max()
    B.close()
    for r in reqs:
        r[0].close()


def test_same_shape_requests_coalesce():
    """Requests of one direction on one plan file, lmax and precision run as
    one transform of their summed maps (gathered and scattered inside the
    graph); every request's output equals its single call bit for bit."""
    from wavemoth_b200.batch import Batch
    rng = np.random.default_rng(77)
    specs = [(32, 1, "split", "alm2map"), (16, 2, "double", "map2alm"), (32, 3, "split", "alm2map"),
             (32, 2, "double", "alm2map"), (16, 1, "double", "map2alm"), (32, 2, "split", "alm2map")]
    reqs, singles = [], []
    for i, (nside, nmaps, prec, direction) in enumerate(specs):
        T = _transform(nside, nmaps, prec)
        if direction == "alm2map":
            inp = torch.from_numpy(osht.random_alm(T.lmax, nmaps, seed=700 + i)).cuda()
            out = torch.full((T.npix, nmaps), float("nan"), dtype=torch.float64, device="cuda")
            single = T.alm2map(inp).clone()
        else:
            inp = torch.from_numpy(rng.standard_normal((T.npix, nmaps))).cuda()
            out = torch.full((T.nalm, nmaps), complex(float("nan"), float("nan")), dtype=torch.complex128,
                             device="cuda")
            single = T.map2alm(inp).clone()
        reqs.append((T, direction, inp, out))
        singles.append(single)
    import tempfile
    B = Batch(reqs, cache=tempfile.mktemp(prefix="wm_sched_", suffix=".json"))
    # three transforms: split alm2map at nside 32 (6 maps), double map2alm at
    # nside 16 (3 maps), double alm2map at nside 32
    assert B.transforms() == 3
    for _ in range(2):
        for r in reqs:
            r[3].fill_(float("nan"))
        B.execute()
        torch.cuda.synchronize()
        for r, s in zip(reqs, singles):
            assert torch.equal(r[3], s)
    for r in reqs:
        r[0].device_status()
    B.close()
    for r in reqs:
        r[0].close()


def test_batch_rejects_shared_transform():
    from wavemoth_b200.batch import Batch
    T = _transform(8, 1, "double")
    a = torch.from_numpy(osht.random_alm(16, 1, seed=1)).cuda()
    m = torch.empty((T.npix, 1), dtype=torch.float64, device="cuda")
    with pytest.raises(ValueError):
        Batch([(T, "alm2map", a, m), (T, "alm2map", a, m)])
    T.close()


def test_uneven_batch_with_nside512_against_reference():
    """A batch holding an nside 512 (lmax 1024) split request next to smaller
    ones: its maps against the reference's own C alm2map of the same alm on
    the same plan file (<= 1e-9 max-abs over max-abs, the split bound), and
    the FP64 request against the same at <= 1e-10."""
    ref = pytest.importorskip("oracle.ref")
    if not ref.available():
        pytest.skip("reference C library not built")
    import os
    import tempfile
    from wavemoth_b200.batch import Batch
    from wavemoth_b200.sht import Transform
    workers = min(len(os.sched_getaffinity(0)), 32)
    big = plan_file(512, 1024, 64, 1e-10, 20.0, workers=workers)
    specs = [(512, 2, "split", big), (512, 1, "double", big), (128, 3, "split", None), (64, 5, "double", None)]
    reqs, alms = [], []
    for i, (nside, nmaps, prec, path) in enumerate(specs):
        path = path or plan_file(nside, 2 * nside, 16, 1e-10, 20.0)
        T = Transform(path, nside, 2 * nside, nmaps, precision=prec)
        a = osht.random_alm(2 * nside, nmaps, seed=900 + i)
        reqs.append((T, "alm2map", torch.from_numpy(a).cuda(),
                     torch.empty((T.npix, nmaps), dtype=torch.float64, device="cuda")))
        alms.append(a)
    B = Batch(reqs, cache=tempfile.mktemp(prefix="wm_sched_", suffix=".json"))
    B.execute()
    torch.cuda.synchronize()
    for (nside, nmaps, prec, path), (T, _, _, out), a in zip(specs, reqs, alms):
        T.device_status()
        if nside != 512:
            continue
        rp = ref.RefPlan(nside, 2 * nside, nmaps, big, nthreads=8)
        rp.input[:] = a
        want = rp.execute().copy()
        rp.close()
        tol = 1e-9 if prec == "split" else 1e-10
        assert np.abs(out.cpu().numpy() - want).max() <= tol * np.abs(want).max()
    B.close()
    for r in reqs:
        r[0].close()
