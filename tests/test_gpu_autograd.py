"""Differentiation through the hand-written kernels (wavemoth_b200.autograd).

* torch.autograd.gradcheck of alm2map and map2alm at nside 4 (full
  numerical Jacobian against the adjoint kernels).
* The differentiable-alm2map workload at nside 256, lmax 512, float64:
  loss = sum_p w_p (alm2map(a)_p - d_p)^2 with seeded w_p ~ U(0.5, 1.5) and
  d = alm2map(a*) + N(0, 0.01^2); central differences at eps = 1e-6 on 64
  random alm entries, and the dot-product test of the backward pass.
* The gradient against a dense one built from the reference's own FP64
  Legendre values (libpshtlight ylmgen through oracle.ref) and the exact
  per-ring DFT adjoint.

Tolerances are stated per test; the loss is quadratic, so central
differences carry rounding error only (|L| eps_mach / eps ~ 1e-8 here).
"""
import math

import numpy as np
import pytest
import torch

from oracle import sht as osht

from .plans import plan_file

pytestmark = pytest.mark.gpu


def _transform(nside, lmax, nmaps, eps=1e-10, chunk=64):
    from wavemoth_b200.sht import Transform
    return Transform(plan_file(nside, lmax, chunk, eps, 20.0, workers=8), nside, lmax, nmaps)


def _dev(x):
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


@pytest.mark.parametrize("nmaps", [1, 2])
def test_gradcheck_alm2map(nmaps):
    from wavemoth_b200.autograd import alm2map
    T = _transform(4, 8, nmaps)
    a = _dev(osht.random_alm(8, nmaps, seed=40 + nmaps)).requires_grad_(True)
    assert torch.autograd.gradcheck(lambda x: alm2map(x, T), (a,), eps=1e-6, atol=1e-8, rtol=1e-6)
    T.close()


def test_gradcheck_map2alm():
    from wavemoth_b200.autograd import map2alm
    T = _transform(4, 8, 2)
    f = _dev(np.random.default_rng(41).standard_normal((192, 2))).requires_grad_(True)
    assert torch.autograd.gradcheck(lambda x: map2alm(x, T), (f,), eps=1e-6, atol=1e-8, rtol=1e-6)
    T.close()


def _config3():
    """Seeded inputs of the nside 256 / lmax 512 differentiable workload."""
    from wavemoth_b200.autograd import alm2map
    nside, lmax = 256, 512
    T = _transform(nside, lmax, 1)
    rng = np.random.default_rng(2025)
    a_star = osht.random_alm(lmax, 1, seed=2026)
    w = _dev(rng.uniform(0.5, 1.5, (T.npix, 1)))
    with torch.no_grad():
        d = T.alm2map(_dev(a_star)) + _dev(rng.normal(0.0, 0.01, (T.npix, 1)))
    a0 = a_star + 0.1 * osht.random_alm(lmax, 1, seed=2027)

    def loss(a):
        return torch.sum(w * (alm2map(a, T) - d) ** 2)

    return T, a0, loss


def test_config3_finite_differences():
    T, a0, loss = _config3()
    a = _dev(a0).requires_grad_(True)
    L = loss(a)
    (g,) = torch.autograd.grad(L, a)
    g = g.cpu().numpy()
    rng = np.random.default_rng(7)
    lmax = T.lmax
    ms = np.concatenate([np.full(lmax - m + 1, m) for m in range(lmax + 1)])
    idx = rng.choice(T.nalm, 64, replace=False)
    eps = 1e-6
    gmax = np.abs(g).max()
    worst = 0.0
    with torch.no_grad():
        for k, i in enumerate(idx):
            part = 1j if (k % 2 and ms[i] > 0) else 1.0
            e = np.zeros_like(a0)
            e[i, 0] = eps * part
            lp = float(loss(_dev(a0 + e)))
            lm = float(loss(_dev(a0 - e)))
            fd = (lp - lm) / (2 * eps)
            an = g[i, 0].imag if part == 1j else g[i, 0].real
            worst = max(worst, abs(fd - an))
    # rounding of the two loss sums over 786k pixels, divided by 2 eps
    assert worst <= 1e-6 * gmax, (worst, gmax)
    T.close()


def test_config3_dot_product():
    """<J v, u> = <v, J^T u> for the alm2map Jacobian J (real inner products)."""
    from wavemoth_b200.autograd import alm2map
    T, a0, _ = _config3()
    a = _dev(a0).requires_grad_(True)
    f = alm2map(a, T)
    u = _dev(np.random.default_rng(8).standard_normal((T.npix, 1)))
    (g,) = torch.autograd.grad(f, a, u)
    v = osht.random_alm(T.lmax, 1, seed=9)
    with torch.no_grad():
        jv = T.alm2map(_dev(v))
    lhs = float(torch.sum(jv * u))
    gn = g.cpu().numpy()
    rhs = float(np.sum(v.real * gn.real + v.imag * gn.imag))
    assert abs(lhs - rhs) <= 1e-11 * np.linalg.norm(jv.cpu().numpy()) * np.linalg.norm(u.cpu().numpy())
    T.close()


def _dense_gradient(nside, lmax, gmap, legendre):
    """grad_a of <alm2map(a), gmap> from Lambda_lm(theta_r) and the ring DFT:
    d f_p / d Re a_lm = c_m Lambda cos(m phi_p), d f_p / d Im a_lm = -c_m Lambda sin(m phi_p)."""
    phi0, offs, _ = osht.grid(nside)
    thetas = osht.ring_thetas(nside)
    nr = thetas.shape[0]
    nmaps = gmap.shape[1]
    S = np.zeros((lmax + 1, nr, nmaps), np.complex128)  # sum_j g e^{-i m phi_j}
    ms = np.arange(lmax + 1)
    for r in range(nr):
        n = offs[r + 1] - offs[r]
        phis = phi0[r] + 2 * np.pi * np.arange(n) / n
        E = np.exp(-1j * np.outer(ms, phis))
        S[:, r, :] = E @ gmap[offs[r]:offs[r + 1]]
    out = np.zeros(((lmax + 1) * (lmax + 2) // 2, nmaps), np.complex128)
    for m in range(lmax + 1):
        L = legendre(m, thetas, lmax)  # (nr, lmax - m + 1)
        c = 1.0 if m == 0 else 2.0
        G = c * (L.T @ S[m])
        o = osht.alm_offset(m, lmax)
        out[o:o + lmax - m + 1] = G.real + (1j * G.imag if m > 0 else 0)
    return out


def test_gradient_against_reference_legendre():
    from oracle import ref
    from wavemoth_b200.autograd import alm2map
    legendre = ref.legendre if ref.available() else osht.normalized_legendre
    nside, lmax, nmaps = 16, 32, 2
    T = _transform(nside, lmax, nmaps, eps=1e-12)
    a = _dev(osht.random_alm(lmax, nmaps, seed=13)).requires_grad_(True)
    gmap = np.random.default_rng(14).standard_normal((T.npix, nmaps))
    (g,) = torch.autograd.grad(alm2map(a, T), a, _dev(gmap))
    want = _dense_gradient(nside, lmax, gmap, legendre)
    got = g.cpu().numpy()
    assert np.linalg.norm(got - want) <= 1e-10 * np.linalg.norm(want)
    T.close()


def test_map2alm_backward_matches_scaled_alm2map():
    """grad_f <map2alm(f), b>_real = (4 pi / Npix) alm2map(b / c_m), Im b_l0 dropped."""
    from wavemoth_b200.autograd import map2alm
    nside, lmax = 8, 16
    T = _transform(nside, lmax, 1)
    f = _dev(np.random.default_rng(15).standard_normal((T.npix, 1))).requires_grad_(True)
    b = osht.random_alm(lmax, 1, seed=16)
    (g,) = torch.autograd.grad(map2alm(f, T), f, _dev(b))
    c = np.concatenate([np.full(lmax - m + 1, 1.0 if m == 0 else 2.0) for m in range(lmax + 1)])
    want = osht.alm2map_dense(nside, b / c[:, None], lmax) * (4 * math.pi / T.npix)
    assert np.linalg.norm(g.cpu().numpy() - want) <= 1e-10 * np.linalg.norm(want)
    T.close()
