"""GPU parity of the CUDA path (through the C ABI) against the oracle and the
reference's own C library on the same plan files and seeded inputs.

Tolerances: plain FP64 results are compared with the reference C library and
the oracle's butterfly restatement at <= 1e-10 relative L2 error (the
acceptance bound for the plain path); the butterfly transform against the
dense exact transform at <= 10 * eps (wavemoth/test/test_wavemoth.py:156).
"""
import hashlib

import numpy as np
import pytest

from oracle import sht as osht
from wavemoth_b200 import lib as wlib
from wavemoth_b200.healpix import lm_to_idx_mmajor

from .plans import plan_file, rel

pytestmark = pytest.mark.gpu

CONFIGS = [
    # nside, lmax, chunk, eps, memop
    (4, 8, 4, 1e-10, 1.0),
    (8, 16, 8, 1e-10, 1.0),
    (16, 32, 8, 1e-10, 1e-10),
    (32, 64, 16, 1e-10, 20.0),
    (32, 32, 32, 1e-11, 1e10),
]


def _alm2map_gpu(path, nside, lmax, alm):
    out = np.zeros((12 * nside * nside, alm.shape[1]))
    inp = np.ascontiguousarray(alm)
    p = wlib.ShtPlan(nside, lmax, lmax, inp, out, "mmajor", matrix_data_filename=path)
    res = p.execute().copy()
    work = p.get_work()
    p.close()
    return res, work


def _map2alm_gpu(path, nside, lmax, maps):
    alm = np.zeros(((lmax + 1) * (lmax + 2) // 2, maps.shape[1]), np.complex128)
    p = wlib.ShtPlan(nside, lmax, lmax, np.ascontiguousarray(maps), alm, "mmajor",
                     matrix_data_filename=path, direction="map2alm")
    res = p.execute().copy()
    p.close()
    return res


@pytest.mark.parametrize("cfg", CONFIGS)
@pytest.mark.parametrize("nmaps", [1, 3])
def test_alm2map_matches_oracle(cfg, nmaps):
    _alm2map_case(cfg, nmaps)


@pytest.mark.parametrize("cfg", [CONFIGS[1], CONFIGS[3]])
@pytest.mark.parametrize("nmaps", [5, 17, 40])
def test_alm2map_many_maps(cfg, nmaps):
    """Vector blocking of the tensor-core path: 10, 34 and 80 real vectors."""
    _alm2map_case(cfg, nmaps)


@pytest.mark.parametrize("cfg", [CONFIGS[1], CONFIGS[3]])
@pytest.mark.parametrize("nmaps", [5, 40])
def test_map2alm_many_maps(cfg, nmaps):
    nside, lmax, chunk, eps, memop = cfg
    path = plan_file(nside, lmax, chunk, eps, memop)
    maps = np.random.default_rng(nmaps).standard_normal((12 * nside * nside, nmaps))
    got = _map2alm_gpu(path, nside, lmax, maps)
    want = osht.map2alm_butterfly(osht.Rev1File(path), maps, lmax)
    assert rel(got, want) < 1e-10


def _alm2map_case(cfg, nmaps):
    nside, lmax, chunk, eps, memop = cfg
    path = plan_file(nside, lmax, chunk, eps, memop)
    alm = osht.random_alm(lmax, nmaps, seed=100 + nmaps)
    got, work = _alm2map_gpu(path, nside, lmax, alm)
    f = osht.Rev1File(path)
    want_work = osht.legendre_phase_butterfly(f, alm, lmax)
    want = osht.backward_ffts(want_work, nside, lmax)
    assert rel(work, want_work) < 1e-12
    assert rel(got, want) < 1e-10
    dense = osht.alm2map_dense(nside, alm, lmax)
    assert rel(got, dense) < 10 * max(eps, 1e-12)


@pytest.mark.parametrize("cfg", CONFIGS[:4])
def test_alm2map_matches_reference_c(cfg):
    ref = pytest.importorskip("oracle.ref")
    if not ref.available():
        pytest.skip("reference C library not built")
    nside, lmax, chunk, eps, memop = cfg
    path = plan_file(nside, lmax, chunk, eps, memop)
    nmaps = 2
    alm = osht.random_alm(lmax, nmaps, seed=7)
    got, work = _alm2map_gpu(path, nside, lmax, alm)
    rp = ref.RefPlan(nside, lmax, nmaps, path, nthreads=2)
    rp.input[:] = alm
    want = rp.execute().copy()
    rp.perform_legendre_transforms()
    want_work = rp.get_work()
    rp.close()
    assert rel(got, want) < 1e-10
    assert rel(work, want_work) < 1e-12


def test_basic_pure_modes():
    """wavemoth/test/test_wavemoth.py:65-90 (assert_basic) against the dense oracle."""
    nside, lmax = 4, 8
    path = plan_file(nside, lmax, 4, 1e-10, 1.0)
    for nmaps in (1, 2, 6, 8):
        alm = np.zeros(((lmax + 1) * (lmax + 2) // 2, nmaps), np.complex128)
        alm[0, :] = 10
        alm[lm_to_idx_mmajor(1, 0, lmax), :] = np.arange(nmaps) * 30
        alm[lm_to_idx_mmajor(2, 1, lmax), :] = 10 + 5j
        got, _ = _alm2map_gpu(path, nside, lmax, alm)
        want = osht.alm2map_dense(nside, alm, lmax)
        np.testing.assert_almost_equal(got, want, 7)


def test_deterministic():
    """wavemoth/test/test_wavemoth.py:92-117: bitwise identical repeats."""
    nside, lmax = 16, 32
    path = plan_file(nside, lmax, 4, 1e-10, 1.0)
    alm = np.zeros(((lmax + 1) * (lmax + 2) // 2, 1), np.complex128)
    alm[lm_to_idx_mmajor(10, 4, lmax)] = 1 + 1j
    out = np.zeros((12 * nside * nside, 1))
    p = wlib.ShtPlan(nside, lmax, lmax, alm, out, "mmajor", matrix_data_filename=path)
    h0 = hashlib.md5(p.execute().tobytes()).hexdigest()
    for _ in range(50):
        assert hashlib.md5(p.execute().tobytes()).hexdigest() == h0
    p.close()


@pytest.mark.parametrize("cfg", CONFIGS)
def test_map2alm_matches_oracle(cfg):
    nside, lmax, chunk, eps, memop = cfg
    path = plan_file(nside, lmax, chunk, eps, memop)
    rng = np.random.default_rng(5)
    maps = rng.standard_normal((12 * nside * nside, 2))
    got = _map2alm_gpu(path, nside, lmax, maps)
    f = osht.Rev1File(path)
    want = osht.map2alm_butterfly(f, maps, lmax)
    assert rel(got, want) < 1e-10
    dense = osht.map2alm_dense(nside, maps, lmax)
    assert rel(got, dense) < 10 * max(eps, 1e-12)


@pytest.mark.parametrize("cfg", CONFIGS[1:4])
def test_dot_product_adjoint(cfg):
    """<alm2map(a), f> = <a, map2alm(f)>_w * Npix / (4 pi) on the GPU path."""
    nside, lmax, chunk, eps, memop = cfg
    path = plan_file(nside, lmax, chunk, eps, memop)
    a = osht.random_alm(lmax, 2, seed=11)
    fmap = np.random.default_rng(12).standard_normal((12 * nside * nside, 2))
    y, _ = _alm2map_gpu(path, nside, lmax, a)
    b = _map2alm_gpu(path, nside, lmax, fmap)
    lhs = float(np.sum(y * fmap))
    rhs = osht.weighted_alm_dot(a, b, lmax) * (12 * nside * nside) / (4 * np.pi)
    assert abs(lhs - rhs) <= 1e-11 * (abs(lhs) + np.linalg.norm(y) * np.linalg.norm(fmap))


def test_config1_nside64_against_reference():
    """Headline configuration 1: plain FP64 alm2map, nside 64, lmax 128, 1 map,
    re/im ~ N(0,1)(l+1)^-1 seeded, plan eps 1e-10 chunk 64: <= 1e-10
    relative to the reference's own FP64 transform."""
    ref = pytest.importorskip("oracle.ref")
    nside, lmax = 64, 128
    path = plan_file(nside, lmax, 64, 1e-10, 20.0)
    alm = osht.random_alm(lmax, 1, seed=2024)
    got, _ = _alm2map_gpu(path, nside, lmax, alm)
    if ref.available():
        rp = ref.RefPlan(nside, lmax, 1, path, nthreads=4)
        rp.input[:] = alm
        want = rp.execute().copy()
        rp.close()
    else:
        want = osht.alm2map_butterfly(osht.Rev1File(path), alm, lmax)
    assert rel(got, want) < 1e-10


def test_config2_nside512_round_trip():
    """Round trip alm2map -> map2alm at nside 512, lmax 1024, 1 map, alm
    re/im ~ N(0,1)(l+1)^-1.5, plan ID eps 1e-12: alm2map within 1e-10 of the
    reference's own C transform (or the oracle's butterfly), map2alm pinned
    to it through the adjoint identity at this size, and the split path's
    map and round trip within 1e-9 of the FP64 ones."""
    import os
    ref = pytest.importorskip("oracle.ref")
    nside, lmax = 512, 1024
    npix = 12 * nside * nside
    path = plan_file(nside, lmax, 64, 1e-12, 20.0, workers=min(os.cpu_count() or 1, 32))
    alm = osht.random_alm(lmax, 1, seed=2, power=1.5)
    maps, _ = _alm2map_gpu(path, nside, lmax, alm)
    if ref.available():
        rp = ref.RefPlan(nside, lmax, 1, path, nthreads=8)
        rp.input[:] = alm
        want = rp.execute().copy()
        rp.close()
        assert rel(maps, want) < 1e-10
    back = _map2alm_gpu(path, nside, lmax, maps)
    f = np.random.default_rng(3).standard_normal((npix, 1))
    b = _map2alm_gpu(path, nside, lmax, f)
    lhs = float(np.sum(maps * f))
    rhs = osht.weighted_alm_dot(alm, b, lmax) * npix / (4 * np.pi)
    assert abs(lhs - rhs) <= 1e-11 * (abs(lhs) + np.linalg.norm(maps) * np.linalg.norm(f))
    out = np.zeros((npix, 1))
    p = wlib.ShtPlan(nside, lmax, lmax, np.ascontiguousarray(alm), out, "mmajor", matrix_data_filename=path,
                     precision="split")
    maps_s = p.execute().copy()
    p.close()
    alm_s = np.zeros_like(alm)
    p = wlib.ShtPlan(nside, lmax, lmax, np.ascontiguousarray(maps_s), alm_s, "mmajor",
                     matrix_data_filename=path, direction="map2alm", precision="split")
    back_s = p.execute().copy()
    p.close()
    assert np.abs(maps_s - maps).max() <= 1e-9 * np.abs(maps).max()
    assert np.abs(back_s - back).max() <= 1e-9 * np.abs(back).max()


def test_depth_capped_plan_matches_reference_c():
    """A plan file written with every matrix capped at one interpolation level
    (the tensor-core paths' depth) against the reference C library on the
    same file, and against the dense transform."""
    ref = pytest.importorskip("oracle.ref")
    if not ref.available():
        pytest.skip("reference C library not built")
    nside, lmax, eps = 128, 256, 1e-10
    path = plan_file(nside, lmax, 64, eps, 1e-10, workers=4, max_levels=1)
    nmaps = 2
    alm = osht.random_alm(lmax, nmaps, seed=11)
    got, work = _alm2map_gpu(path, nside, lmax, alm)
    rp = ref.RefPlan(nside, lmax, nmaps, path, nthreads=2)
    rp.input[:] = alm
    want = rp.execute().copy()
    rp.close()
    assert rel(got, want) < 1e-10
    dense = osht.alm2map_dense(nside, alm, lmax)
    assert rel(got, dense) < 10 * eps
