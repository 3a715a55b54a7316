"""Plan-file writer: butterfly compression of the per-(m, parity) Legendre
matrices and the rev1 resource-file format read by the plan.

This is the precompute step of the reference (wavemoth/lib.pyx:301-592,
wavemoth/butterfly.pyx:527-825, scripts/precompute.py), restated:

* ``butterfly_compress`` builds the same tree as butterfly.pyx:537-680: the
  columns (rings) are cut into chunks of ``chunk_size`` (padded with empty
  chunks to a power of two), then pairs of neighbouring column blocks are
  joined, split vertically into a top (T) and bottom (B) half, and each half
  is replaced by an interpolative decomposition to precision ``eps``.
* the level at which the tree is cut into roots is chosen by the same cost
  model (lib.pyx:518-543): interpolation elements plus residual elements
  weighted by (5/2 + 1)/memop_cost.
* residual blocks (the "D" factor) are stored as Legendre-recurrence strips
  (lib.pyx:397-486 with stripify at :301-368), each strip holding x^2 and the
  two starting rows; blocks of at most 4 rows are stored dense.
* the binary layout is rev1 (src/wavemoth.c:203-264, src/butterfly.c.in:
  434-445, src/butterfly.h.in:8-88), byte for byte.

Differences from the reference writer that do not change the format:
the ID is this library's own pivoted-QR implementation (wm_host_interp_decomp,
same stopping rule as iddp_id), the Legendre values come from this library's
generator, and each residual payload is written once (butterfly.pyx:798-804
writes the payload list n+1 times; only the last copy is referenced).
"""
import io
import os
import struct
from concurrent.futures import ProcessPoolExecutor
import multiprocessing as mp

import numpy as np

from . import _native
from .healpix import get_ring_thetas

RESOURCE_FORMAT_VERSION = 1


# --------------------------------------------------------------------------
# stream helpers (wavemoth/streamutils.pyx:1-25)
# --------------------------------------------------------------------------

def _pad16(stream):
    r = stream.tell() % 16
    if r:
        stream.write(b"\0" * (16 - r))


def _i32(stream, v):
    stream.write(struct.pack("<i", int(v)))


def _i64(stream, v):
    stream.write(struct.pack("<q", int(v)))


def _raw(stream, arr, order="C"):
    stream.write(np.asarray(arr).tobytes(order=order))


def _aligned(stream, arr, order="C"):
    _pad16(stream)
    _raw(stream, arr, order)


# --------------------------------------------------------------------------
# tree
# --------------------------------------------------------------------------

class ResidualBlock:
    """Rows [row_start, row_stop) of the matrix restricted to col_indices."""
    __slots__ = ("row_start", "row_stop", "col_indices")

    def __init__(self, row_start, row_stop, col_indices):
        self.row_start = int(row_start)
        self.row_stop = int(row_stop)
        self.col_indices = np.asarray(col_indices, dtype=np.int64)


class InterpolationBlock:
    """k x n matrix [I_k | T] with column permutation given by filter:
    filter[j] == 0 for the k skeleton columns (identity part), 1 otherwise."""

    def __init__(self, filter, interpolant):
        self.filter = np.ascontiguousarray(filter, dtype=np.int8)
        self.interpolant = np.asfortranarray(interpolant, dtype=np.float64)
        n = self.filter.shape[0]
        k = n - int(self.filter.sum())
        if self.interpolant.shape != (k, n - k):
            raise ValueError("interpolant shape %r does not match filter (k=%d, n=%d)"
                             % (self.interpolant.shape, k, n))
        self.k, self.n = k, n

    def size(self):
        return self.interpolant.size + self.filter.shape[0]

    def apply(self, x):
        """y = A x (butterfly.pyx:258-264)."""
        y = x[self.filter == 0, :].copy()
        y += self.interpolant @ x[self.filter == 1, :]
        return y

    def transpose_apply(self, x):
        """y = A^T x (butterfly.pyx:266-274)."""
        y = np.empty((self.n, x.shape[1]))
        y[self.filter == 0, :] = x
        y[self.filter == 1, :] = self.interpolant.T @ x
        return y

    def as_array(self):
        out = np.zeros((self.k, self.n))
        out[:, self.filter == 0] = np.eye(self.k)
        out[:, self.filter == 1] = self.interpolant
        return out


class IdentityNode:
    def __init__(self, n, remainder_blocks=None):
        self.ncols = self.node_ncols = self.node_nrows = int(n)
        self.block_heights = [int(n)]
        if remainder_blocks is None:
            remainder_blocks = [ResidualBlock(0, n, np.zeros(0, np.int64))]
        self.remainder_blocks = remainder_blocks
        self.nrows = remainder_blocks[0].row_stop - remainder_blocks[0].row_start
        self.children = []
        self.blocks = []

    def get_max_depth(self):
        return 0

    def get_k_max(self):
        return self.ncols

    def get_nblocks_max(self):
        return 1

    def size(self):
        return 0

    def get_nodes_at_level(self, level):
        if level == 0:
            return [self]
        raise ValueError("level too high")

    def get_stats(self, level=None, residual_size_func=None):
        if level not in (0, None):
            raise ValueError("level too high")
        f = residual_size_func or (lambda a, b: a * b)
        size = f(self.nrows, self.ncols)
        return size, 0, size


class InnerNode:
    def __init__(self, blocks, children, remainder_blocks=None):
        L, R = children
        for (T, B), lh, rh in zip(blocks, L.block_heights, R.block_heights):
            if not (T.n == B.n == lh + rh):
                raise ValueError("nonconforming interpolation blocks")
        self.blocks = blocks
        self.children = [L, R]
        self.ncols = L.ncols + R.ncols
        self.node_ncols = L.node_nrows + R.node_nrows
        self.block_heights = [h for T, B in blocks for h in (T.k, B.k)]
        self.node_nrows = sum(self.block_heights)
        if remainder_blocks is None:
            # a bare interpolation node (butterfly.pyx:326-329)
            remainder_blocks = [ResidualBlock(0, h, np.zeros(0, np.int64))
                                for h in self.block_heights]
            self.nrows = self.node_nrows
        else:
            if len(remainder_blocks) != len(self.block_heights):
                raise ValueError("remainder_blocks has wrong length")
            self.nrows = sum(r.row_stop - r.row_start for r in remainder_blocks)
        self.remainder_blocks = remainder_blocks

    def get_max_depth(self):
        return 1 + max(c.get_max_depth() for c in self.children)

    def get_k_max(self):
        return max([max(self.block_heights)] + [c.get_k_max() for c in self.children])

    def get_nblocks_max(self):
        return len(self.block_heights)

    def size(self):
        return (sum(c.size() for c in self.children)
                + sum(T.size() + B.size() for T, B in self.blocks))

    def get_nodes_at_level(self, level):
        if level == 0:
            return [self]
        return [n for c in self.children for n in c.get_nodes_at_level(level - 1)]

    def get_stats(self, level=None, residual_size_func=None):
        """(uncompressed, interpolation, residual) element counts when the
        tree is cut `level` levels above the leaves (butterfly.pyx:501-524)."""
        f = residual_size_func or (lambda a, b: a * b)
        depth = self.get_max_depth()
        if level is None:
            level = depth
        if self.nrows == 0 or self.ncols == 0:
            return 0, 0, 0
        if level == 0:
            size = f(self.nrows, self.ncols)
            return size, 0, size
        nodes = self.get_nodes_at_level(depth - level)
        res = sum(f(r.row_stop - r.row_start, len(r.col_indices))
                  for node in nodes for r in node.remainder_blocks)
        ip = sum(node.size() for node in nodes)
        return self.nrows * self.ncols, ip, res


def make_partition(start, stop, chunk_size):
    """End column of every chunk (butterfly.pyx:633-640)."""
    n = stop - start
    result = list(range(chunk_size, n, chunk_size))
    if len(result) == 0 or result[-1] != stop:
        result.append(stop)
    return result


def pad_with_empty_columns(partition):
    """Repeat ends (empty chunks) until the count is a power of two
    (butterfly.pyx:619-631)."""
    n = len(partition)
    target = 1
    while n > target:
        target *= 2
    to_add = target - n
    result = []
    for p in partition:
        result.append(p)
        if to_add > 0:
            result.append(p)
            to_add -= 1
    return result


def permutations_to_filter(iden, ipol):
    f = np.zeros(len(iden) + len(ipol), dtype=np.int8)
    f[np.asarray(ipol, dtype=np.int64)] = 1
    return f


def sparse_interpolative_decomposition(A, eps):
    """(iden, ipol, A_ip) with A[:, ipol] ~= A[:, iden] @ A_ip, both index lists
    sorted (interpolative_decomposition.pyx:182-247)."""
    m, n = A.shape
    if n == 0:
        return np.zeros(0, np.int64), np.zeros(0, np.int64), np.zeros((0, 0))
    if m == 0:
        return np.zeros(0, np.int64), np.arange(n), np.zeros((0, n))
    k, perm, proj = _native.interp_decomp(A, eps)
    iden, ipol = perm[:k], perm[k:]
    o = np.argsort(ipol, kind="stable")
    proj = proj[:, o]
    ipol = ipol[o]
    o = np.argsort(iden, kind="stable")
    proj = proj[o, :]
    iden = iden[o]
    return iden, ipol, proj


def butterfly_compress(provider, chunk_size, shape=None, eps=1e-10):
    """Butterfly tree of the (nrows, ncols) matrix served by provider.get_block
    (an ndarray is wrapped in an ArrayProvider)."""
    if isinstance(provider, np.ndarray):
        if shape is None:
            shape = provider.shape
        provider = ArrayProvider(provider)
    elif shape is None:
        raise TypeError("shape must be provided")
    nrows, ncols = shape
    partition = pad_with_empty_columns(make_partition(0, ncols, chunk_size))

    def core(col, part):
        if len(part) == 1:
            stop = part[0]
            cols = np.arange(col, stop)
            blk = provider.get_block(0, nrows, cols)
            return [blk], IdentityNode(stop - col, [ResidualBlock(0, nrows, cols)])
        mid = len(part) // 2
        Lk, Ln = core(col, part[:mid])
        Rk, Rn = core(col + Ln.ncols, part[mid:])
        rems, pairs, kept = [], [], []
        for Lr, Rr, Lb, Rb in zip(Ln.remainder_blocks, Rn.remainder_blocks, Lk, Rk):
            cols = np.concatenate([Lr.col_indices, Rr.col_indices])
            LR = np.hstack([Lb, Rb])
            vmid = LR.shape[0] // 2
            pair = []
            row = Lr.row_start
            for X in (LR[:vmid, :], LR[vmid:, :]):
                iden, ipol, A_ip = sparse_interpolative_decomposition(X, eps)
                pair.append(InterpolationBlock(permutations_to_filter(iden, ipol), A_ip))
                rems.append(ResidualBlock(row, row + X.shape[0], cols[iden]))
                kept.append(np.asfortranarray(X[:, iden]))
                row += X.shape[0]
            pairs.append(tuple(pair))
        return kept, InnerNode(pairs, (Ln, Rn), rems)

    return core(0, partition)[1]


# --------------------------------------------------------------------------
# heap layout and serialisation (butterfly.pyx:682-825)
# --------------------------------------------------------------------------

def heapify(root, skip_levels=0):
    """Nodes of the forest cut `skip_levels` below root, in binary-heap order:
    roots at indices [0, 2^skip), children of heap slot s (1-based position
    p = s + 2^skip) at positions 2p, 2p+1."""
    K = root.get_max_depth()
    heap = [None] * (2 ** (K + 1) - 2 ** skip_levels)
    nroots = 2 ** skip_levels

    def forest(node, s):
        return [node] if s == 0 else [x for c in node.children for x in forest(c, s - 1)]

    def place(node, pos):
        heap[pos - nroots] = node
        for i, c in enumerate(node.children):
            place(c, 2 * pos + i)

    for i, r in enumerate(forest(root, skip_levels)):
        place(r, nroots + i)
    return heap


def _serialize_node(stream, node):
    if isinstance(node, InnerNode):
        _i32(stream, len(node.block_heights))
        _raw(stream, np.asarray(node.block_heights, dtype=np.int32))
        for T, B in node.blocks:
            for blk in (T, B):
                _raw(stream, blk.filter)
                _pad16(stream)
                _raw(stream, blk.interpolant, order="F")
    else:
        _i32(stream, 0)
        _i32(stream, node.ncols)


def serialize_butterfly_matrix(root, provider, num_levels=None, stream=None):
    if stream is None:
        stream = io.BytesIO()
    start = stream.tell()
    if start % 16:
        raise ValueError("stream must be 16-byte aligned")
    depth = root.get_max_depth()
    if num_levels is None:
        num_levels = depth
    elif num_levels == 0:
        root = IdentityNode(root.ncols, [ResidualBlock(0, root.nrows, np.arange(root.ncols))])
        depth = num_levels = 0
    skip = max(0, depth - num_levels)
    nroots = 2 ** skip
    heap = heapify(root, skip)
    forest = heap[:nroots]
    k_max = 0 if depth == 0 else max(r.get_k_max() for r in forest)
    nblocks_max = max(r.get_nblocks_max() for r in forest)

    _i32(stream, forest[0].nrows)
    _i32(stream, root.ncols)
    _i32(stream, k_max)
    _i32(stream, nblocks_max)
    _i64(stream, root.size())
    _i32(stream, nroots)
    _i32(stream, len(heap))
    _i32(stream, nroots)
    _i32(stream, 0)
    residual_table = stream.tell()
    for _ in range(nroots):
        _i64(stream, 0)
    heap_table = stream.tell()
    for _ in heap:
        _i64(stream, 0)

    for i, node in enumerate(forest):
        pos = stream.tell()
        stream.seek(residual_table + 8 * i)
        _i64(stream, pos - start)
        stream.seek(pos)
        nb = len(node.remainder_blocks)
        _i64(stream, nb)
        offsets_pos = stream.tell()
        for _ in range(nb + 1):
            _i64(stream, 0)
        offs = []
        for r in node.remainder_blocks:
            offs.append(stream.tell())
            provider.serialize_block_payload(stream, r.row_start, r.row_stop, r.col_indices)
        offs.append(stream.tell())
        end = stream.tell()
        stream.seek(offsets_pos)
        for o in offs:
            _i64(stream, o - start)
        stream.seek(end)

    node_offsets = []
    for node in heap:
        _pad16(stream)
        node_offsets.append(stream.tell())
        _serialize_node(stream, node)
    end = stream.tell()
    stream.seek(heap_table)
    for o in node_offsets:
        _i64(stream, o - start)
    stream.seek(end)
    return stream


class ArrayProvider:
    """Serves blocks of an in-memory matrix; payloads are dense column-major
    blocks (butterfly.pyx:642-658)."""

    def __init__(self, array):
        self.array = np.asarray(array, dtype=np.float64)

    def get_block(self, row_start, row_stop, col_indices):
        if len(col_indices) > 0:
            return self.array[row_start:row_stop][:, col_indices]
        return np.zeros((row_stop - row_start, 0))

    def serialize_block_payload(self, stream, row_start, row_stop, col_indices):
        _pad16(stream)
        _i64(stream, row_start)
        _i64(stream, row_stop)
        _raw(stream, self.get_block(row_start, row_stop, col_indices), order="F")


# --------------------------------------------------------------------------
# Legendre matrix provider (lib.pyx:301-486)
# --------------------------------------------------------------------------

def _first_true(x):
    nz = np.flatnonzero(x)
    return nz[0] if nz.shape[0] else x.shape[0]


def stripify(A, include_above=1e-30, exclude_below=1e-80, jump_treshold=10, col_divisor=6):
    """Greedy partition of a matrix whose columns grow in magnitude
    downwards into strips (row_start, row_stop, col_start, col_stop) that
    keep every element >= include_above and drop every element < exclude_below
    (lib.pyx:301-368)."""
    inc = np.log2(include_above)
    exc = np.log2(exclude_below)
    M = np.array(A, dtype=np.float64, order="F")
    zero = (M == 0)
    M[zero] = 1
    M = np.log2(np.abs(M))
    M[zero] = exc - 1
    nrows, ncols = M.shape
    above_exc = M >= exc
    above_inc = M >= inc
    starts = []
    for c in range(ncols):
        a = _first_true(above_exc[:, c])
        b = _first_true(above_inc[:, c])
        if np.any(~above_exc[a:, c]):
            raise ValueError("Magnitude of column %d not increasing regularly enough" % c)
        starts.append((a, b))
    inf = nrows + 1
    max_a, min_b, start_col = -1, inf, 0
    strips = []
    starts.append((inf, inf))
    for c, (a, b) in enumerate(starts):
        needed = a > min_b or b < max_a
        wanted = c > 0 and (b - min_b) > jump_treshold
        if needed or (wanted and c % col_divisor == 0):
            strips.append((min_b, nrows, start_col, c))
            start_col = c
            max_a, min_b = a, b
        max_a = max(a, max_a)
        min_b = min(b, min_b)
    return strips


class LegendreMatrixProvider:
    """Even (odd=0) or odd (odd=1) rows l = m + 2k + odd of Lambda_m, columns
    = the 2*nside northern rings from the equator (lib.pyx:376-395)."""

    def __init__(self, m, odd, nside, lmax, check_stability=True):
        self.m, self.odd, self.lmax = m, odd, lmax
        self.thetas = get_ring_thetas(nside, positive_only=True)
        self.x2 = np.cos(self.thetas) ** 2
        self.ncols_full_matrix = self.thetas.shape[0]
        self.nk = max(0, (lmax - m - odd) // 2 + 1)
        self.check_stability = check_stability
        if self.nk > 0:
            full = _native.legendre_matrix(m, self.thetas, lmax, 1e-300)  # (ni, lmax-m+1)
            # the eps=1e-30 variant zeroes everything before the first
            # |lambda| > 1e-30 (per ring, scanning all l)
            first = np.argmax(np.abs(full) > 1e-30, axis=1)
            first[~np.any(np.abs(full) > 1e-30, axis=1)] = full.shape[1]
            cut = full.copy()
            cut[np.arange(full.shape[1])[None, :] < first[:, None]] = 0.0
            self.L300 = np.ascontiguousarray(full.T[odd::2, :])   # (nk, ni)
            self.L30 = np.ascontiguousarray(cut.T[odd::2, :])
        else:
            self.L300 = self.L30 = np.zeros((0, self.ncols_full_matrix))

    def row_to_l(self, row):
        return self.m + 2 * row + self.odd

    def get_block(self, row_start, row_stop, col_indices):
        return self.L30[row_start:row_stop][:, col_indices]

    def serialize_block_payload(self, stream, row_start, row_stop, col_indices):
        col_indices = np.asarray(col_indices, dtype=np.int64)
        if len(col_indices) == 0 or row_start == row_stop:
            _pad16(stream)
            _i64(stream, 0)
            _i64(stream, 0)
            return
        lmin = self.row_to_l(row_start)
        x2 = self.x2[col_indices]
        Lam = self.L300[row_start:row_stop][:, col_indices]
        strips = stripify(Lam, include_above=1e-30, exclude_below=1e-250,
                          jump_treshold=10, col_divisor=6)
        shift = min(s[0] for s in strips)
        row_start += shift
        lmin += 2 * shift
        Lam = Lam[shift:, :]
        strips = [(a - shift, b - shift, c, d) for a, b, c, d in strips]
        _pad16(stream)
        _i64(stream, row_start)
        _i64(stream, row_stop)
        nk = row_stop - row_start
        if nk <= 4:
            _aligned(stream, Lam, order="F")
            return
        _i64(stream, len(strips))
        aux = _native.recurrence_coefficients(self.m, lmin, nk)
        _aligned(stream, aux)
        prev = 0
        for rstart, rstop, cstart, cstop in strips:
            assert rstop == nk and cstart == prev
            prev = cstop
            _i64(stream, rstart)
            _i64(stream, cstop)
            if rstop - rstart <= 4:
                _aligned(stream, Lam[rstart:rstop, cstart:cstop], order="F")
            else:
                P0 = np.ascontiguousarray(Lam[rstart, cstart:cstop])
                P1 = np.ascontiguousarray(Lam[rstart + 1, cstart:cstop])
                xs = np.ascontiguousarray(x2[cstart:cstop])
                _aligned(stream, xs)
                _aligned(stream, P0)
                _aligned(stream, P1)
                if self.check_stability:
                    y = _native.recurrence_last_row(xs, P0, P1, aux[3 * rstart:], rstop - rstart)
                    ny = np.linalg.norm(y)
                    if ny > 0 and np.linalg.norm(y - Lam[-1, cstart:cstop]) / ny > 1e-9:
                        raise ArithmeticError("numerically unstable recurrence start "
                                              "(m=%d, rows %d..%d)" % (self.m, row_start, row_stop))
        assert prev == Lam.shape[1]


# --------------------------------------------------------------------------
# whole resource file
# --------------------------------------------------------------------------

class ResourceComputer:
    """Writes a rev1 resource file for (nside, lmax, mmax)
    (lib.pyx:512-592)."""

    def __init__(self, nside, lmax, mmax, chunk_size=64, eps=1e-10, memop_cost=20.0,
                 check_stability=True, max_levels=None):
        if lmax != mmax:
            raise ValueError("only lmax == mmax is supported")
        if max_levels is not None and max_levels < 0:
            raise ValueError("max_levels must be None or >= 0")
        self.nside, self.lmax, self.mmax = nside, lmax, mmax
        self.chunk_size, self.eps, self.memop_cost = chunk_size, eps, memop_cost
        self.check_stability = check_stability
        # None: every depth the tree has (the reference's choice); else the
        # level choice stops at this many interpolation levels -- 1 keeps
        # every matrix on this library's tensor-core paths, which run trees
        # of depth 0 and 1 (deeper ones run on the generic FP64 kernels)
        self.max_levels = max_levels

    def residual_cost(self, rows, cols):
        return rows * cols * (5.0 / 2.0 + 1) / self.memop_cost

    def compute_matrix(self, m, odd):
        provider = LegendreMatrixProvider(m, odd, self.nside, self.lmax, self.check_stability)
        tree = butterfly_compress(provider, self.chunk_size,
                                  shape=(provider.nk, provider.ncols_full_matrix), eps=self.eps)
        depth = tree.get_max_depth()
        if self.max_levels is not None:
            depth = min(depth, self.max_levels)
        costs = np.zeros(depth + 1)
        for level in range(depth + 1):
            _, ip, res = tree.get_stats(level, self.residual_cost)
            costs[level] = ip + res
        best = int(costs.argmin())
        return serialize_butterfly_matrix(tree, provider, num_levels=best).getvalue()

    def compute(self, stream, max_workers=1):
        _i64(stream, self.lmax)
        _i64(stream, self.mmax)
        _i64(stream, self.nside)
        header = stream.tell()
        for _ in range(4 * (self.mmax + 1)):
            _i64(stream, 0)
        jobs = [(m, odd) for m in range(self.mmax + 1) for odd in (0, 1)]
        if max_workers <= 1:
            results = (_compute_one(self, m, odd) for m, odd in jobs)
            self._write_all(stream, header, jobs, results)
        else:
            ctx = mp.get_context("spawn")
            with ProcessPoolExecutor(max_workers=max_workers, mp_context=ctx) as ex:
                # submit in chunks so that memory stays bounded
                futs = [ex.submit(_compute_one, self, m, odd) for m, odd in jobs]
                self._write_all(stream, header, jobs, (f.result() for f in futs))
        return stream

    def _write_all(self, stream, header, jobs, results):
        for (m, odd), data in zip(jobs, results):
            _pad16(stream)
            pos = stream.tell()
            stream.write(data)
            end = stream.tell()
            stream.seek(header + (4 * m + 2 * odd) * 8)
            _i64(stream, pos)
            _i64(stream, end - pos)
            stream.seek(end)


def _compute_one(rc, m, odd):
    return rc.compute_matrix(m, odd)


def compute_resource_file(path, nside, lmax, mmax=None, chunk_size=64, eps=1e-10,
                          memop_cost=20.0, max_workers=None, max_levels=None):
    """Write a rev1 plan file for (nside, lmax) to `path`; returns path.
    max_levels caps the interpolation levels of every matrix (None: the
    cost model's choice over all of them)."""
    mmax = lmax if mmax is None else mmax
    if max_workers is None:
        max_workers = min(32, len(os.sched_getaffinity(0)))
    rc = ResourceComputer(nside, lmax, mmax, chunk_size, eps, memop_cost, max_levels=max_levels)
    tmp = path + ".tmp%d" % os.getpid()
    with open(tmp, "wb") as f:
        rc.compute(f, max_workers=max_workers)
    os.replace(tmp, path)
    return path


def query_resourcefile(path):
    """(nside, lmax) from a rev1 header (src/wavemoth.c:144-155)."""
    with open(path, "rb") as f:
        head = f.read(24)
    if len(head) < 24:
        raise ValueError("truncated resource file header: %s" % path)
    lmax, mmax, nside = struct.unpack("<qqq", head)
    return nside, lmax


def default_resource_path(resource_dir, nside):
    """<dir>/rev1/<nside>.dat (src/wavemoth.c:137-142)."""
    return os.path.join(resource_dir, "rev%d" % RESOURCE_FORMAT_VERSION, "%d.dat" % nside)
