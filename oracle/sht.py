"""ORACLE (test infrastructure only): CPU restatement of the reference's
alm2map path, its map2alm adjoint, and readers for the rev1 plan format.

Every function cites the reference code whose behaviour it restates.  The
scalar Legendre pieces live in oracle/legendre.c (built into
oracle/_build/liboracle.so by oracle/Makefile).

map2alm has no reference implementation (the reference is synthesis only);
here it is defined as (4 pi / Npix) times the adjoint of alm2map with respect
to the real inner product on maps and the inner product
<a, b> = sum_lm c_m Re(a_lm conj(b_lm)), c_0 = 1, c_m = 2 (m > 0), on alm;
i.e. a_lm = (4 pi / Npix) sum_p f_p lambda_lm(theta_p) e^{-i m phi_p}.
"""
import ctypes
import os
import struct
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def _lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "_build", "liboracle.so")
        if not os.path.exists(path):
            subprocess.run(["make", "-C", _HERE, "all"], check=True, capture_output=True)
        lib = ctypes.CDLL(path)
        dp = ctypes.POINTER(ctypes.c_double)
        lib.or_normalized_legendre.argtypes = [ctypes.c_int, dp, ctypes.c_int, ctypes.c_int,
                                               ctypes.c_double, dp]
        lib.or_normalized_legendre.restype = ctypes.c_int
        lib.or_legendre_auxdata.argtypes = [ctypes.c_int64] * 3 + [dp]
        lib.or_legendre_auxdata.restype = None
        for name in ("or_legendre_transform", "or_legendre_transform_T"):
            fn = getattr(lib, name)
            fn.argtypes = [ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, dp, ctypes.c_int64,
                           dp, dp, dp, dp, dp]
            fn.restype = None
        _LIB = lib
    return _LIB


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


# ---------------------------------------------------------------- geometry
# wavemoth/healpix.py:5-40 and src/wavemoth.c:1199-1232

def ring_thetas(nside, positive_only=False):
    nr = 4 * nside - 1 if not positive_only else 2 * nside
    i = np.arange(1, nr + 1, dtype=np.float64)
    z = np.empty(nr)
    z[:nside] = 1 - i[:nside] ** 2 / (3 * nside ** 2)
    z[nside:2 * nside] = 4.0 / 3.0 - (2 * i[nside:2 * nside]) / (3 * nside)
    if positive_only:
        return np.arccos(z[::-1])
    z[2 * nside:] = -z[2 * nside - 2::-1]
    return np.arccos(z)


def grid(nside):
    """(phi0[nrings], ring_offsets[nrings+1], mid_ring) as src/wavemoth.c:1199-1232."""
    nr = 4 * nside - 1
    phi0 = np.empty(nr)
    offs = np.empty(nr + 1, np.int64)
    npix_ring = 0
    ipix = 0
    for r in range(nr):
        if r <= nside - 1:
            npix_ring += 4
            phi0[r] = np.pi / (4.0 * (r + 1))
        elif r > 3 * nside - 1:
            npix_ring -= 4
            phi0[r] = np.pi / (4.0 * (nr - r))
        else:
            phi0[r] = (np.pi / (4.0 * nside)) * (r % 2)
        offs[r] = ipix
        ipix += npix_ring
    offs[nr] = ipix
    return phi0, offs, 2 * nside - 1


def alm_offset(m, lmax):
    return m * (2 * lmax - m + 3) // 2


# ---------------------------------------------------------------- Legendre

def normalized_legendre(m, thetas, lmax, epsilon=1e-300):
    """(ntheta, lmax-m+1), wavemoth/legendre.pyx:24-57."""
    th = np.ascontiguousarray(thetas, dtype=np.float64)
    out = np.empty((th.shape[0], lmax - m + 1))
    rc = _lib().or_normalized_legendre(int(m), _dp(th), th.shape[0], int(lmax), float(epsilon),
                                      _dp(out))
    if rc != 0:
        raise ValueError("or_normalized_legendre: %d" % rc)
    return out


def legendre_auxdata(m, lmin, nk):
    if nk < 3:
        return np.zeros(0)
    out = np.empty(3 * (nk - 2))
    _lib().or_legendre_auxdata(int(m), int(lmin), int(nk), _dp(out))
    return out


def legendre_transform(a_packed, x2, aux, P0, P1):
    """y (nx, nvecs) = P^T a for the strip recurrence (legendre_transform.c.in:680-716)."""
    a = np.ascontiguousarray(a_packed, dtype=np.float64)
    nk, nvecs = a.shape
    nx = x2.shape[0]
    y = np.zeros((nx, nvecs))
    aux = np.ascontiguousarray(aux, dtype=np.float64) if len(aux) else np.zeros(1)
    _lib().or_legendre_transform(nx, nk, nvecs, _dp(a), nvecs, _dp(y),
                                 _dp(np.ascontiguousarray(x2)), _dp(aux),
                                 _dp(np.ascontiguousarray(P0)), _dp(np.ascontiguousarray(P1)))
    return y


def legendre_transform_T(y, nk, x2, aux, P0, P1):
    """a (nk, nvecs) = P y, the adjoint of legendre_transform."""
    y = np.ascontiguousarray(y, dtype=np.float64)
    nx, nvecs = y.shape
    a = np.zeros((nk, nvecs))
    aux = np.ascontiguousarray(aux, dtype=np.float64) if len(aux) else np.zeros(1)
    _lib().or_legendre_transform_T(nx, nk, nvecs, _dp(a), nvecs, _dp(y),
                                   _dp(np.ascontiguousarray(x2)), _dp(aux),
                                   _dp(np.ascontiguousarray(P0)), _dp(np.ascontiguousarray(P1)))
    return a


# ---------------------------------------------------------------- rev1 files

def _pad16(pos):
    return pos + (-pos) % 16


class Payload:
    """A decoded residual payload (src/wavemoth.c:958-1009; writer
    wavemoth/lib.pyx:397-486)."""

    def __init__(self, buf, off, ncols):
        off = _pad16(off)
        self.row_start, self.row_stop = struct.unpack_from("<qq", buf, off)
        off += 16
        nk = self.row_stop - self.row_start
        self.ncols = ncols
        self.dense = None
        self.strips = []
        if nk <= 4 or ncols == 0:
            off = _pad16(off)
            self.dense = np.frombuffer(buf, np.float64, nk * ncols, off).reshape((nk, ncols), order="F")
            return
        (nstrips,) = struct.unpack_from("<q", buf, off)
        off += 8
        off = _pad16(off)
        self.aux = np.frombuffer(buf, np.float64, 3 * (nk - 2), off)
        off += 8 * 3 * (nk - 2)
        cstart = 0
        for _ in range(nstrips):
            rstart, cstop = struct.unpack_from("<qq", buf, off)
            off += 16
            nx = cstop - cstart
            nks = nk - rstart
            if nks <= 4:
                off = _pad16(off)
                A = np.frombuffer(buf, np.float64, nks * nx, off).reshape((nks, nx), order="F")
                off += 8 * nks * nx
                self.strips.append((rstart, cstart, cstop, "dense", A))
            else:
                arrs = []
                for _k in range(3):
                    off = _pad16(off)
                    arrs.append(np.frombuffer(buf, np.float64, nx, off))
                    off += 8 * nx
                self.strips.append((rstart, cstart, cstop, "rec", tuple(arrs)))
            cstart = cstop

    def pull(self, a_packed):
        """buf (ncols, nvecs) = D^T a for this block; a_packed rows are the
        matrix rows (every other l)."""
        nvecs = a_packed.shape[1]
        out = np.zeros((self.ncols, nvecs))
        a = a_packed[self.row_start:self.row_stop]
        if self.dense is not None:
            if self.dense.size:
                out[:] = self.dense.T @ a
            return out
        for rstart, cstart, cstop, kind, data in self.strips:
            if kind == "dense":
                out[cstart:cstop] = data.T @ a[rstart:]
            else:
                x2, P0, P1 = data
                out[cstart:cstop] = legendre_transform(a[rstart:], x2, self.aux[3 * rstart:], P0, P1)
        return out

    def push(self, x, a_packed):
        """a_packed[rows] += D x (the map2alm direction)."""
        if self.dense is not None:
            if self.dense.size:
                a_packed[self.row_start:self.row_stop] += self.dense @ x
            return
        a = a_packed[self.row_start:self.row_stop]
        for rstart, cstart, cstop, kind, data in self.strips:
            if kind == "dense":
                a[rstart:] += data @ x[cstart:cstop]
            else:
                x2, P0, P1 = data
                a[rstart:] += legendre_transform_T(x[cstart:cstop], a.shape[0] - rstart, x2,
                                                   self.aux[3 * rstart:], P0, P1)


class Matrix:
    """One butterfly-compressed (m, parity) matrix (format:
    src/butterfly.h.in:8-88, reader src/butterfly.c.in:284-445)."""

    def __init__(self, buf, base):
        self.buf, self.base = buf, base
        (self.nrows, self.ncols, self.k_max, self.nblocks_max, self.element_count,
         self.first_level_size, self.heap_size, self.heap_first_index, _) = \
            struct.unpack_from("<iiiiqiiii", buf, base)
        off = base + 40
        self.residual_offsets = struct.unpack_from("<%dq" % self.first_level_size, buf, off)
        off += 8 * self.first_level_size
        self.node_offsets = struct.unpack_from("<%dq" % self.heap_size, buf, off)

    def node(self, pos):
        """(nblocks, block_heights, data offset after the heights) of heap position pos."""
        off = self.base + self.node_offsets[pos - self.heap_first_index]
        (nb,) = struct.unpack_from("<i", self.buf, off)
        off += 4
        if nb == 0:
            (n,) = struct.unpack_from("<i", self.buf, off)
            return 0, [n], None
        bh = list(struct.unpack_from("<%di" % nb, self.buf, off))
        return nb, bh, off + 4 * nb

    def _interp_blocks(self, pos):
        """Yields (i, j, k, n_left, n_right, filter, interpolant) in storage order."""
        nb, bh, off = self.node(pos)
        _, lbh, _ = self.node(2 * pos)
        _, rbh, _ = self.node(2 * pos + 1)
        for i in range(nb // 2):
            nl, nr = lbh[i], rbh[i]
            n = nl + nr
            for j in range(2):
                k = bh[2 * i + j]
                filt = np.frombuffer(self.buf, np.int8, n, off)
                off = _pad16(off + n)
                ip = np.frombuffer(self.buf, np.float64, k * (n - k), off).reshape((k, n - k), order="F")
                off += 8 * k * (n - k)
                yield i, j, k, nl, nr, filt, ip

    def payloads(self, root):
        off = self.base + self.residual_offsets[root]
        (n,) = struct.unpack_from("<q", self.buf, off)
        offs = struct.unpack_from("<%dq" % (n + 1), self.buf, off + 8)
        return [self.base + o for o in offs]

    # ---- alm2map Legendre step: q = A^T a  (butterfly.c.in:284-432) ----
    def transpose_apply(self, a_packed):
        nvecs = a_packed.shape[1]
        q = np.zeros((self.ncols, nvecs))
        start = 0
        for r in range(self.first_level_size):
            pos = self.heap_first_index + r
            pl = self.payloads(r)
            nb, bh, _ = self.node(pos)
            if nb == 0:
                pay = Payload(self.buf, pl[0], bh[0])
                q[start:start + bh[0]] = pay.pull(a_packed)
                start += bh[0]
            else:
                inputs = [Payload(self.buf, pl[j], bh[j]).pull(a_packed) for j in range(nb)]
                start = self._t_node(pos, start, inputs, q)
        assert start == self.ncols
        return q

    def transpose_apply_rows(self, x):
        """y = A^T x where the residual factor is the identity: root block j
        takes rows [pos, pos + k_j) of x in order (the pull of
        ButterflyPlan.transpose_pull_input, butterfly.pyx:134-141)."""
        nvecs = x.shape[1]
        q = np.zeros((self.ncols, nvecs))
        start = 0
        pos_in = 0
        for r in range(self.first_level_size):
            pos = self.heap_first_index + r
            nb, bh, _ = self.node(pos)
            if nb == 0:
                q[start:start + bh[0]] = x[pos_in:pos_in + bh[0]]
                pos_in += bh[0]
                start += bh[0]
            else:
                inputs = []
                for j in range(nb):
                    inputs.append(x[pos_in:pos_in + bh[j]])
                    pos_in += bh[j]
                start = self._t_node(pos, start, inputs, q)
        return q

    def _t_node(self, pos, start, inputs, q):
        nb, bh, _ = self.node(pos)
        if nb == 0:
            n = bh[0]
            q[start:start + n] = inputs[0]
            return start + n
        outs_l, outs_r = [], []
        acc = None
        for i, j, k, nl, nr, filt, ip in self._interp_blocks(pos):
            x = inputs[2 * i + j]
            z = np.empty((nl + nr, x.shape[1]))
            z[filt == 0] = x
            z[filt == 1] = ip.T @ x
            acc = z if j == 0 else acc + z
            if j == 1:
                outs_l.append(acc[:nl])
                outs_r.append(acc[nl:])
        start = self._t_node(2 * pos, start, outs_l, q)
        return self._t_node(2 * pos + 1, start, outs_r, q)

    # ---- map2alm Legendre step: a = A q  (butterfly.pyx:372-405 and the
    #      transpose of the residual pull) ----
    def apply(self, q, nk_total):
        nvecs = q.shape[1]
        a = np.zeros((nk_total, nvecs))
        start = 0
        for r in range(self.first_level_size):
            pos = self.heap_first_index + r
            pl = self.payloads(r)
            nb, bh, _ = self.node(pos)
            if nb == 0:
                Payload(self.buf, pl[0], bh[0]).push(q[start:start + bh[0]], a)
                start += bh[0]
            else:
                blocks, start = self._f_node(pos, start, q)
                for j in range(nb):
                    Payload(self.buf, pl[j], bh[j]).push(blocks[j], a)
        return a

    def _f_node(self, pos, start, q):
        """Returns this node's output blocks (one per block height) and the
        next column."""
        nb, bh, _ = self.node(pos)
        if nb == 0:
            n = bh[0]
            return [q[start:start + n]], start + n
        left, start = self._f_node(2 * pos, start, q)
        right, start = self._f_node(2 * pos + 1, start, q)
        out = []
        for i, j, k, nl, nr, filt, ip in self._interp_blocks(pos):
            z = np.vstack([left[i], right[i]])
            out.append(z[filt == 0] + ip @ z[filt == 1])
        return out, start


class Rev1File:
    """A rev1 resource file (src/wavemoth.c:203-264)."""

    def __init__(self, path_or_bytes):
        if isinstance(path_or_bytes, (bytes, bytearray)):
            self.buf = bytes(path_or_bytes)
        else:
            with open(path_or_bytes, "rb") as f:
                self.buf = f.read()
        self.lmax, self.mmax, self.nside = struct.unpack_from("<qqq", self.buf, 0)
        self.offsets = struct.unpack_from("<%dq" % (4 * (self.mmax + 1)), self.buf, 24)

    def matrix(self, m, odd):
        start = self.offsets[4 * m + 2 * odd]
        if start == 0:
            return None
        return Matrix(self.buf, start)


# ---------------------------------------------------------------- transforms

def _packed_rows(alm_m, odd):
    """a rows l = m + odd + 2k of one m (the every-other-row stride of
    src/wavemoth.c:1017-1018) as a real (nk, 2*nmaps) array."""
    sub = np.ascontiguousarray(alm_m[odd::2])
    return sub.view(np.float64).reshape(sub.shape[0], 2 * alm_m.shape[1])


def legendre_phase_butterfly(f, alm, lmax):
    """work[m, odd, ring, map] complex, the Legendre phase of
    wavemoth_execute computed from the plan file f."""
    nmaps = alm.shape[1]
    ni = 2 * f.nside
    work = np.zeros((lmax + 1, 2, ni, nmaps), np.complex128)
    for m in range(lmax + 1):
        o = alm_offset(m, lmax)
        alm_m = alm[o:o + lmax - m + 1]
        for odd in range(2):
            mat = f.matrix(m, odd)
            if mat is None:
                continue
            a = _packed_rows(alm_m, odd)
            q = mat.transpose_apply(a)
            work[m, odd] = q.view(np.complex128).reshape(ni, nmaps)
    return work


def legendre_phase_dense(nside, alm, lmax, epsilon=1e-300):
    """The same work array from dense Lambda (no compression)."""
    nmaps = alm.shape[1]
    th = ring_thetas(nside, positive_only=True)
    work = np.zeros((lmax + 1, 2, 2 * nside, nmaps), np.complex128)
    for m in range(lmax + 1):
        L = normalized_legendre(m, th, lmax, epsilon)  # (ni, nl)
        o = alm_offset(m, lmax)
        alm_m = alm[o:o + lmax - m + 1]
        for odd in range(2):
            work[m, odd] = L[:, odd::2] @ alm_m[odd::2]
    return work


def backward_ffts(work, nside, mmax, phase_shifts=True):
    """Ring assembly and c2r (src/wavemoth.c:1083-1191): map (npix, nmaps)."""
    nmaps = work.shape[3]
    phi0, offs, mid = grid(nside)
    if not phase_shifts:
        phi0 = np.zeros_like(phi0)
    out = np.zeros((offs[-1], nmaps))
    ms = np.arange(mmax + 1)
    for r in range(mid + 1):
        n = offs[mid + r + 1] - offs[mid + r]
        ph = phi0[mid + r]
        shift = (np.cos(ms * ph) + 1j * np.sin(ms * ph))[:, None]
        qe, qo = work[:, 0, r, :], work[:, 1, r, :]
        top = (qe + qo) * shift
        bot = (qe - qo) * shift
        j1 = ms % n
        j2 = (n - ms) % n
        for W_src, ring_off in ((top, offs[mid - r]), (bot, offs[mid + r])):
            if r == 0 and ring_off == offs[mid + r] and W_src is bot:
                continue
            W = np.zeros((n // 2 + 1, nmaps), np.complex128)
            ok1 = j1 <= n // 2
            np.add.at(W, j1[ok1], W_src[ok1])
            ok2 = (ms != 0) & (j2 <= n // 2)
            np.add.at(W, j2[ok2], np.conj(W_src[ok2]))
            out[ring_off:ring_off + n] = np.fft.irfft(W, n, axis=0) * n
    return out


def forward_ffts(maps, nside, mmax, scale=None):
    """Adjoint of backward_ffts (up to the c_m weights) times scale
    (default 4 pi / Npix): work~[m, odd, ring, map]."""
    nmaps = maps.shape[1]
    phi0, offs, mid = grid(nside)
    npix = offs[-1]
    if scale is None:
        scale = 4 * np.pi / npix
    work = np.zeros((mmax + 1, 2, mid + 1, nmaps), np.complex128)
    ms = np.arange(mmax + 1)
    for r in range(mid + 1):
        n = offs[mid + r + 1] - offs[mid + r]
        ph = phi0[mid + r]
        unshift = (np.cos(ms * ph) - 1j * np.sin(ms * ph))[:, None]

        def fold(ring):
            F = np.fft.rfft(ring, axis=0)
            j = ms % n
            g = np.where((j <= n // 2)[:, None], F[np.minimum(j, n // 2)],
                         np.conj(F[np.minimum((n - j) % n, n // 2)]))
            return g * unshift * scale

        gt = fold(maps[offs[mid - r]:offs[mid - r] + n])
        if r == 0:
            work[:, 0, r] = gt
            work[:, 1, r] = gt
        else:
            gb = fold(maps[offs[mid + r]:offs[mid + r] + n])
            work[:, 0, r] = gt + gb
            work[:, 1, r] = gt - gb
    return work


def legendre_phase_adjoint_dense(nside, work, lmax, epsilon=1e-300):
    """alm (nalm, nmaps) = sum_rings Lambda work~ (no compression)."""
    nmaps = work.shape[3]
    th = ring_thetas(nside, positive_only=True)
    alm = np.zeros(((lmax + 1) * (lmax + 2) // 2, nmaps), np.complex128)
    for m in range(lmax + 1):
        L = normalized_legendre(m, th, lmax, epsilon)
        o = alm_offset(m, lmax)
        for odd in range(2):
            alm[o + odd:o + lmax - m + 1:2] = L[:, odd::2].T @ work[m, odd]
    return alm


def legendre_phase_adjoint_butterfly(f, work, lmax):
    nmaps = work.shape[3]
    ni = 2 * f.nside
    alm = np.zeros(((lmax + 1) * (lmax + 2) // 2, nmaps), np.complex128)
    for m in range(lmax + 1):
        o = alm_offset(m, lmax)
        for odd in range(2):
            mat = f.matrix(m, odd)
            nk = max(0, (lmax - m - odd) // 2 + 1)
            if mat is None or nk == 0:
                continue
            q = np.ascontiguousarray(work[m, odd]).view(np.float64).reshape(ni, 2 * nmaps)
            a = mat.apply(q, nk)
            alm[o + odd:o + lmax - m + 1:2] = a.view(np.complex128).reshape(nk, nmaps)
    return alm


def alm2map_dense(nside, alm, lmax):
    return backward_ffts(legendre_phase_dense(nside, alm, lmax), nside, lmax)


def alm2map_butterfly(f, alm, lmax):
    return backward_ffts(legendre_phase_butterfly(f, alm, lmax), f.nside, lmax)


def map2alm_dense(nside, maps, lmax):
    return legendre_phase_adjoint_dense(nside, forward_ffts(maps, nside, lmax), lmax)


def map2alm_butterfly(f, maps, lmax):
    return legendre_phase_adjoint_butterfly(f, forward_ffts(maps, f.nside, lmax), lmax)


def weighted_alm_dot(a, b, lmax):
    """<a, b> = sum_lm c_m Re(a_lm conj(b_lm)), c_0 = 1, c_m = 2."""
    w = np.concatenate([np.full(lmax - m + 1, 1.0 if m == 0 else 2.0) for m in range(lmax + 1)])
    return float(np.sum(w[:, None] * np.real(a * np.conj(b))))


def random_alm(lmax, nmaps, seed, power=1.0):
    """re, im iid N(0,1) * (l+1)^-power, Im = 0 at m = 0; m-major layout."""
    rng = np.random.default_rng(seed)
    ls = np.concatenate([np.arange(m, lmax + 1) for m in range(lmax + 1)])
    ms = np.concatenate([np.full(lmax - m + 1, m) for m in range(lmax + 1)])
    re = rng.standard_normal((ls.shape[0], nmaps))
    im = rng.standard_normal((ls.shape[0], nmaps))
    im[ms == 0] = 0
    return ((re + 1j * im) * ((ls + 1.0) ** -power)[:, None]).astype(np.complex128)
