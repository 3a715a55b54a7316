"""Split-precision (sliced int8 tensor-core) residual products against the
plain FP64 path on the same plans and inputs.

Tolerance: the maximum absolute difference over the output, relative to the
maximum magnitude of the FP64 result, at most 1e-9 (the split-precision
acceptance bound); the FP64 path itself is pinned to the reference at 1e-10
in test_gpu_parity.py.  Plans cover depth-0 and depth-1 butterfly trees,
1, 5 and 40 maps (80 vectors: two passes of 64), both directions.
"""
import numpy as np
import pytest

from oracle import sht as osht
from wavemoth_b200 import lib as wlib

from .plans import plan_file

pytestmark = pytest.mark.gpu

CONFIGS = [
    # nside, lmax, chunk, eps, memop
    (8, 16, 8, 1e-10, 1.0),
    (16, 32, 8, 1e-10, 1e-10),
    (32, 64, 16, 1e-10, 20.0),
    (64, 128, 64, 1e-10, 20.0),
]


def maxrel(got, want):
    return float(np.abs(got - want).max() / np.abs(want).max())


def _run(path, nside, lmax, inp, direction, precision):
    if direction == "alm2map":
        out = np.zeros((12 * nside * nside, inp.shape[1]))
    else:
        out = np.zeros(((lmax + 1) * (lmax + 2) // 2, inp.shape[1]), np.complex128)
    p = wlib.ShtPlan(nside, lmax, lmax, np.ascontiguousarray(inp), out, "mmajor",
                     matrix_data_filename=path, direction=direction, precision=precision)
    res = p.execute().copy()
    p.close()
    return res


@pytest.mark.parametrize("cfg", CONFIGS)
@pytest.mark.parametrize("nmaps", [1, 5, 40])
def test_split_alm2map(cfg, nmaps):
    nside, lmax, chunk, eps, memop = cfg
    path = plan_file(nside, lmax, chunk, eps, memop)
    alm = osht.random_alm(lmax, nmaps, seed=300 + nmaps)
    ref = _run(path, nside, lmax, alm, "alm2map", "double")
    got = _run(path, nside, lmax, alm, "alm2map", "split")
    assert maxrel(got, ref) <= 1e-9


@pytest.mark.parametrize("cfg", CONFIGS)
@pytest.mark.parametrize("nmaps", [1, 40])
def test_split_map2alm(cfg, nmaps):
    nside, lmax, chunk, eps, memop = cfg
    path = plan_file(nside, lmax, chunk, eps, memop)
    maps = np.random.default_rng(400 + nmaps).standard_normal((12 * nside * nside, nmaps))
    ref = _run(path, nside, lmax, maps, "map2alm", "double")
    got = _run(path, nside, lmax, maps, "map2alm", "split")
    assert maxrel(got, ref) <= 1e-9


def test_split_against_oracle_and_status():
    """Split alm2map against the oracle's butterfly transform; the device
    status word stays clear."""
    import torch
    from wavemoth_b200.sht import Transform
    nside, lmax = 32, 64
    path = plan_file(nside, lmax, 16, 1e-10, 20.0)
    alm = osht.random_alm(lmax, 3, seed=17)
    T = Transform(path, nside, lmax, 3, precision="split")
    got = T.alm2map(torch.from_numpy(alm).cuda()).cpu().numpy()
    T.device_status()
    want = osht.alm2map_butterfly(osht.Rev1File(path), alm, lmax)
    assert maxrel(got, want) <= 1e-9
    T.close()


@pytest.mark.parametrize("cfg", CONFIGS)
def test_split_stored_equals_generated(cfg):
    """Residual P sliced once per plan (streamed GEMM) and regenerated in the
    GEMM kernels at every call give the same slices, the same int32
    accumulators and so bitwise the same outputs, both directions."""
    nside, lmax, chunk, eps, memop = cfg
    path = plan_file(nside, lmax, chunk, eps, memop)
    alm = osht.random_alm(lmax, 40, seed=500)
    maps = np.random.default_rng(501).standard_normal((12 * nside * nside, 40))
    for direction, inp in (("alm2map", alm), ("map2alm", maps)):
        stored = _run(path, nside, lmax, inp, direction, "split")
        generated = _run(path, nside, lmax, inp, direction, "split-generate")
        assert np.array_equal(stored, generated), direction


@pytest.mark.parametrize("cfg", [CONFIGS[2], CONFIGS[3], (128, 256, 64, 1e-10, 20.0)])
@pytest.mark.parametrize("precision", ["split", "split-generate", "double"])
def test_repeated_calls_alternating_directions(cfg, precision):
    """alm2map, map2alm, alm2map, map2alm on one plan (q and the X buffer
    shared by both directions, outputs prefilled with NaN): every call
    recomputes every output row, so the repeats equal the first calls
    bitwise, and the split results stay within 1e-9 of the FP64 ones.
    High-m columns with no active ring rows (zero tiles) are in these plans."""
    torch = pytest.importorskip("torch")
    from wavemoth_b200.sht import Transform
    nside, lmax, chunk, eps, memop = cfg
    nmaps = 3
    path = plan_file(nside, lmax, chunk, eps, memop)
    alm = torch.from_numpy(osht.random_alm(lmax, nmaps, seed=31)).cuda()
    T = Transform(path, nside, lmax, nmaps, precision=precision)
    P = Transform(path, nside, lmax, nmaps, precision="double")
    want_map = P.alm2map(alm)
    want_alm = P.map2alm(want_map)

    def nan_like(x):
        return torch.full_like(x, float("nan"))

    maps = [T.alm2map(alm, out=nan_like(want_map))]
    alms = [T.map2alm(maps[0], out=nan_like(want_alm))]
    maps.append(T.alm2map(alm, out=nan_like(want_map)))
    alms.append(T.map2alm(maps[1], out=nan_like(want_alm)))
    torch.cuda.synchronize()
    T.device_status()
    for x in maps + alms:
        assert bool(torch.isfinite(x).all())
    assert torch.equal(maps[0], maps[1])
    assert torch.equal(alms[0], alms[1])
    tol = 1e-9 if precision != "double" else 0.0
    assert float((maps[1] - want_map).abs().max()) <= tol * float(want_map.abs().max())
    assert float((alms[1] - want_alm).abs().max()) <= tol * float(want_alm.abs().max())
    T.close()
    P.close()
