"""End-to-end CPU checks of the oracle transforms on plan files written by
the package's writer, against the reference's own C library."""
import hashlib

import numpy as np
import pytest

from oracle import sht as osht
from wavemoth_b200.healpix import lm_to_idx_mmajor

from .plans import plan_file, rel


def ref_or_skip():
    from oracle import ref
    if not ref.available():
        pytest.skip("reference C library not available")
    return ref


@pytest.mark.parametrize("cfg", [(4, 8, 4, 1e-10, 1.0), (16, 32, 8, 1e-10, 1e-10),
                                 (32, 64, 16, 1e-10, 20.0)])
def test_oracle_matches_reference_execute(cfg):
    ref = ref_or_skip()
    nside, lmax, chunk, eps, memop = cfg
    path = plan_file(nside, lmax, chunk, eps, memop)
    alm = osht.random_alm(lmax, 2, seed=1)
    rp = ref.RefPlan(nside, lmax, 2, path, nthreads=2)
    rp.input[:] = alm
    want = rp.execute().copy()
    rp.perform_legendre_transforms()
    want_work = rp.get_work()
    rp.close()
    f = osht.Rev1File(path)
    assert rel(osht.alm2map_butterfly(f, alm, lmax), want) < 1e-13
    assert rel(osht.legendre_phase_butterfly(f, alm, lmax), want_work) < 1e-13


def test_reference_legendre_phase_vs_dense():
    """wavemoth/test/test_wavemoth.py:204-230."""
    ref = ref_or_skip()
    nside, lmax, nmaps = 4, 8, 2
    path = plan_file(nside, lmax, 4, 1e-10, 1.0)
    rp = ref.RefPlan(nside, lmax, nmaps, path, nthreads=3)
    k = np.arange(1, 3)
    for l in range(lmax + 1):
        for m in range(l, lmax + 1):
            rp.input[lm_to_idx_mmajor(l, m, lmax), :] = 10 * k * np.cos(l * 0.1) * np.sqrt(m)
    rp.input[1, :] = (5 + 5j) * k
    rp.input[2, :] = 34 + 3j
    rp.perform_legendre_transforms()
    work = rp.get_work()
    alm = rp.input.copy()
    rp.close()
    work0 = osht.legendre_phase_dense(nside, alm, lmax, epsilon=1e-30)
    np.testing.assert_almost_equal(work0, work)


@pytest.mark.parametrize("eps,memop,nmaps", [(1e-7, 1.0, 1), (1e-11, 1.0, 1), (1e-11, 1e10, 1),
                                             (1e-11, 1e-10, 1), (1e-11, 1e-10, 3)])
def test_accuracy_against_dense(eps, memop, nmaps):
    """wavemoth/test/test_wavemoth.py:123-163 with the dense FP64 oracle in
    place of libpsht: pure modes at the first and last 100 alm indices and
    random maps, max relative error < 10 eps."""
    ref = ref_or_skip()
    nside = lmax = 32
    path = plan_file(nside, lmax, 32, eps, memop)
    rp = ref.RefPlan(nside, lmax, nmaps, path, nthreads=2)
    nalm = rp.input.shape[0]
    errors = []
    for idx in list(range(100)) + list(range(nalm - 100, nalm)):
        rp.input[:] = 0
        rp.input[idx, :] = 1 + 2j * np.arange(1, nmaps + 1)
        got = rp.execute().copy()
        want = osht.alm2map_dense(nside, rp.input.copy(), lmax)
        errors.append(rel(got, want))
    rng = np.random.default_rng(0)
    for _ in range(5):
        rp.input[:] = rng.standard_normal(rp.input.shape) + 1j * rng.standard_normal(rp.input.shape)
        got = rp.execute().copy()
        errors.append(rel(got, osht.alm2map_dense(nside, rp.input.copy(), lmax)))
    rp.close()
    assert max(errors) < 10 * eps


def test_reference_deterministic():
    """wavemoth/test/test_wavemoth.py:92-117."""
    ref = ref_or_skip()
    nside, lmax = 16, 32
    path = plan_file(nside, lmax, 4, 1e-10, 1.0)
    rp = ref.RefPlan(nside, lmax, 1, path, nthreads=4)
    rp.input[lm_to_idx_mmajor(10, 4, lmax)] = 1 + 1j
    h0 = hashlib.md5(rp.execute().tobytes()).hexdigest()
    for _ in range(20):
        assert hashlib.md5(rp.execute().tobytes()).hexdigest() == h0
    rp.close()


@pytest.mark.parametrize("cfg", [(8, 16, 8, 1e-10, 1.0), (16, 32, 8, 1e-10, 1e-10)])
def test_map2alm_definition(cfg):
    """map2alm = (4 pi / Npix) adjoint of alm2map: dot-product identity for
    the dense and the butterfly oracle, and butterfly vs dense."""
    nside, lmax, chunk, eps, memop = cfg
    path = plan_file(nside, lmax, chunk, eps, memop)
    f = osht.Rev1File(path)
    a = osht.random_alm(lmax, 2, seed=5)
    g = np.random.default_rng(6).standard_normal((12 * nside * nside, 2))
    npix = 12 * nside * nside
    for fwd, adj in ((lambda x: osht.alm2map_dense(nside, x, lmax),
                      lambda y: osht.map2alm_dense(nside, y, lmax)),
                     (lambda x: osht.alm2map_butterfly(f, x, lmax),
                      lambda y: osht.map2alm_butterfly(f, y, lmax))):
        lhs = float(np.sum(fwd(a) * g))
        rhs = osht.weighted_alm_dot(a, adj(g), lmax) * npix / (4 * np.pi)
        assert abs(lhs - rhs) < 1e-11 * abs(lhs) + 1e-11
    assert rel(osht.map2alm_butterfly(f, g, lmax), osht.map2alm_dense(nside, g, lmax)) < 10 * eps


def test_writer_deterministic():
    import io
    from wavemoth_b200 import resource
    outs = []
    for _ in range(2):
        s = io.BytesIO()
        resource.ResourceComputer(8, 16, 16, 4, 1e-10, 1.0).compute(s, max_workers=1)
        outs.append(s.getvalue())
    assert outs[0] == outs[1]
