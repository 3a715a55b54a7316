"""Differentiable spherical harmonic transforms (torch.autograd.Function).

alm2map is the real-linear map A from the alm (complex128, m-major, the real
and imaginary parts of every (l, m >= 0) entry as independent real variables;
Im a_l0 does not enter) to the RING-ordered map.  The hand-written map2alm
kernels compute the adjoint transform with the weighted inner product of the
real field,

    map2alm = (4 pi / Npix) W^-1 A^T,   W = diag(c_m), c_0 = 1, c_m = 2,

so the gradients of both directions are one call of the other direction's
kernels with a per-m weight (no Legendre values are stored: the backward
pass regenerates them with the same recurrence as the forward pass):

    alm2map backward:  grad_alm = (Npix / 4 pi) c_m map2alm(grad_map)
    map2alm backward:  grad_map = (4 pi / Npix) alm2map(grad_alm / c_m)

For complex tensors torch expects grad = dL/dRe + i dL/dIm, which is the
componentwise real gradient above.  Im a_l0 gets a zero gradient (the forward
transform ignores it).  The forward definitions follow src/wavemoth.c:1011-1191
(alm2map) and its adjoint; map2alm has no reference implementation.
"""
import math

import torch

from .sht import Transform


def _m_weights(lmax, device):
    """c_m per alm row of the m-major layout (1 at m = 0, else 2)."""
    w = torch.full(((lmax + 1) * (lmax + 2) // 2,), 2.0, dtype=torch.float64, device=device)
    w[: lmax + 1] = 1.0
    return w


class _Alm2Map(torch.autograd.Function):
    @staticmethod
    def forward(ctx, alm, transform):
        ctx.transform = transform
        return transform.alm2map(alm)

    @staticmethod
    def backward(ctx, grad_map):
        T = ctx.transform
        g = T.map2alm(grad_map.contiguous())
        w = _m_weights(T.lmax, g.device) * (T.npix / (4.0 * math.pi))
        g = g * w[:, None]
        g[: T.lmax + 1] = g[: T.lmax + 1].real.to(torch.complex128)
        return g, None


class _Map2Alm(torch.autograd.Function):
    @staticmethod
    def forward(ctx, maps, transform):
        ctx.transform = transform
        return transform.map2alm(maps)

    @staticmethod
    def backward(ctx, grad_alm):
        T = ctx.transform
        w = _m_weights(T.lmax, grad_alm.device)
        g = (grad_alm / w[:, None]).contiguous()
        # Im of m = 0 rows is not an output of map2alm: drop its cotangent
        g[: T.lmax + 1] = g[: T.lmax + 1].real.to(torch.complex128)
        out = T.alm2map(g)
        return out * (4.0 * math.pi / T.npix), None


def alm2map(alm, transform):
    """Differentiable alm2map on `transform` (a wavemoth_b200.sht.Transform)."""
    return _Alm2Map.apply(alm, transform)


def map2alm(maps, transform):
    """Differentiable map2alm on `transform`."""
    return _Map2Alm.apply(maps, transform)


class SphericalHarmonics(torch.nn.Module):
    """Module holding one device plan; forward(alm) -> map, inverse(map) -> alm,
    both differentiable."""

    def __init__(self, resource_file, nside, lmax, nmaps=1):
        super().__init__()
        self.transform = Transform(resource_file, nside, lmax, nmaps)

    def forward(self, alm):
        return alm2map(alm, self.transform)

    def inverse(self, maps):
        return map2alm(maps, self.transform)
