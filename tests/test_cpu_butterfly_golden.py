"""Golden butterfly cases of wavemoth/test/test_butterfly.py, restated: the
package's tree classes and rev1 serializer, applied by the oracle's
restatement and by the reference's own C bfm_transpose_apply_d."""
import io

import numpy as np
import pytest

from oracle import sht as osht
from wavemoth_b200.resource import (ArrayProvider, IdentityNode, InnerNode, InterpolationBlock,
                                    butterfly_compress, heapify, make_partition,
                                    permutations_to_filter, serialize_butterfly_matrix, stripify)


class NoPayload:
    """test_butterfly.py:111-116."""

    def get_block(self, *a):
        raise AssertionError("no payload")

    def serialize_block_payload(self, stream, row_start, row_stop, col_indices):
        return


def ref_or_skip():
    from oracle import ref
    if not ref.available():
        pytest.skip("reference C library not available")
    return ref


def vectors(m, n):
    """test_butterfly.py:104-109."""
    x = np.arange(1, m + 1)
    return np.stack([x * 10 ** i for i in range(n)], axis=1).astype(np.float64)


def ndrange(shape, start=0):
    return np.arange(start, np.prod(shape) + start, dtype=np.float64).reshape(shape)


def both_applies(node, x):
    data = serialize_butterfly_matrix(node, NoPayload()).getvalue()
    mat = osht.Matrix(data, 0)
    y_oracle = mat.transpose_apply_rows(x)
    ref = ref_or_skip()
    y_ref = ref.bfm_transpose_apply(data, x, mode="rows")
    return y_oracle, y_ref


def test_permutations_to_filter():
    assert list(permutations_to_filter([2, 3, 5], [0, 4])) == [1, 0, 0, 0, 1]
    assert list(permutations_to_filter([0, 1, 2], [])) == [0, 0, 0]
    assert list(permutations_to_filter([], [0, 1])) == [1, 1]
    assert list(permutations_to_filter([], [])) == []


def test_make_partition():
    assert make_partition(0, 22, 10) == [10, 20, 22]
    assert make_partition(0, 12, 10) == [10, 12]
    assert make_partition(0, 10, 10) == [10]
    assert make_partition(0, 9, 10) == [9]
    assert make_partition(0, 0, 10) == [0]


class _N:
    def __init__(self, value, children=()):
        self.value, self.children = value, list(children)

    def get_max_depth(self):
        return 0 if not self.children else 1 + max(c.get_max_depth() for c in self.children)


def _vals(heap):
    return [None if h is None else h.value for h in heap]


def test_heapify():
    """test_butterfly.py:70-99 (complete trees)."""
    t = _N(0, [_N(1, [_N(3), _N(4)]), _N(2, [_N(5), _N(6)])])
    assert _vals(heapify(t)) == [0, 1, 2, 3, 4, 5, 6]
    assert _vals(heapify(_N(10))) == [10]
    assert _vals(heapify(t, skip_levels=1)) == [1, 2, 3, 4, 5, 6]
    assert _vals(heapify(t, skip_levels=2)) == [3, 4, 5, 6]


def test_transpose_apply_leaf():
    node = IdentityNode(7)
    x = ndrange((7, 2))
    yo, yr = both_applies(node, x)
    assert np.array_equal(yo, x) and np.array_equal(yr, x)


def test_transpose_apply_small_fullrank():
    A = np.array([[1, 0], [0, 1], [1, 0], [0, 1]], dtype=np.float64)
    S1 = InnerNode([(InterpolationBlock([0, 0], np.zeros((2, 0))),
                     InterpolationBlock([0, 0], np.zeros((2, 0))))],
                   [IdentityNode(1), IdentityNode(1)])
    x = vectors(4, 2)
    yo, yr = both_applies(S1, x)
    assert np.array_equal(yo, A.T @ x) and np.array_equal(yr, A.T @ x)


def test_transpose_apply_small_zerorank():
    S1 = InnerNode([(InterpolationBlock([1, 1], np.zeros((0, 2))),
                     InterpolationBlock([1, 1], np.zeros((0, 2))))],
                   [IdentityNode(1), IdentityNode(1)])
    yo, yr = both_applies(S1, np.ones((0, 2)))
    assert yo.shape == (2, 2) and np.all(yo == 0) and np.all(yr == 0)


def test_transpose_apply_small_ip():
    """The exact interpolating golden matrix of test_butterfly.py:172-186."""
    A = np.array([[1, 0, 10], [0, 1, 100], [1, -1, 0], [0, -2, 1]], dtype=np.float64)
    S1 = InnerNode([(InterpolationBlock([0, 0, 1], [[10], [100]]),
                     InterpolationBlock([0, 1, 0], [[-1], [-2]]))],
                   [IdentityNode(1), IdentityNode(2)])
    x = vectors(4, 2)
    yo, yr = both_applies(S1, x)
    assert np.array_equal(yo, A.T @ x) and np.array_equal(yr, A.T @ x)


def test_transpose_apply_tree_generated():
    """Deep generated tree (test_butterfly.py:188-249): oracle and reference
    C agree exactly, and both equal the dense product of the tree's blocks."""
    nextk = [1]

    def make_tree(n):
        if n == 0:
            k = nextk[0]
            nextk[0] += 1
            return IdentityNode(k)
        L, R = make_tree(n // 2), make_tree(n // 2)
        blocks = []
        for lh, rh in zip(L.block_heights, R.block_heights):
            nn = lh + rh
            TB = []
            for k in (max(1, nn - 4), max(1, nn - 3)):
                f = np.ones(nn, np.int8)
                f[:k] = 0
                TB.append(InterpolationBlock(f, ndrange((k, nn - k), start=3)))
            blocks.append(tuple(TB))
        return InnerNode(blocks, [L, R])

    root = make_tree(4)
    x = ndrange((root.nrows, 2))
    yo, yr = both_applies(root, x)
    assert np.array_equal(yo, yr)
    # dense: apply the transpose to the identity, column by column
    eye = np.eye(root.nrows)
    At = osht.Matrix(serialize_butterfly_matrix(root, NoPayload()).getvalue(), 0).transpose_apply_rows(eye)
    np.testing.assert_allclose(yo, At @ x, rtol=1e-13)


@pytest.mark.parametrize("num_levels", [1, 2, 200])
def test_transpose_apply_dense_residual(num_levels):
    """test_butterfly.py:370-389: A = i*j (20 x 10), chunk 3, residual
    payloads dense, embedded at a 160-byte stream offset."""
    ref = ref_or_skip()
    i, j = np.ogrid[:20, :10]
    A = (i * j).astype(np.float64)
    tree = butterfly_compress(A, chunk_size=3)
    stream = io.BytesIO()
    stream.write(b"a" * 160)
    data = serialize_butterfly_matrix(tree, ArrayProvider(A), stream=stream,
                                      num_levels=num_levels).getvalue()[160:]
    x = ndrange((20, 2))
    y = ref.bfm_transpose_apply(data, x, mode="dense")
    np.testing.assert_allclose(y, A.T @ x, rtol=1e-12, atol=1e-9)


@pytest.mark.parametrize("chunk", range(1, 10))
def test_compress_roundtrip(chunk):
    """test_butterfly.py:294-313: compress and uncompress reproduce A."""
    ref = ref_or_skip()
    A = ndrange((10, 10), start=1)
    tree = butterfly_compress(A, chunk)
    data = serialize_butterfly_matrix(tree, ArrayProvider(A)).getvalue()
    At = ref.bfm_transpose_apply(data, np.eye(10), mode="dense")
    np.testing.assert_allclose(At.T, A, rtol=1e-9, atol=1e-9)


def test_stripify_golden():
    """test_wavemoth.py:170-177."""
    A = np.ones((2, 3))
    assert stripify(A) == [(0, 2, 0, 3)]
    A[0, 1] = 0
    assert stripify(A) == [(0, 2, 0, 1), (1, 2, 1, 2), (0, 2, 2, 3)]
    A += 1
    A[:, 2] = 0
    assert stripify(A) == [(0, 2, 0, 2), (2, 2, 2, 3)]


@pytest.mark.parametrize("nside,m", [(32, 40), (256, 270), (256, 271)])
def test_stripify_legendre(nside, m):
    """test_wavemoth.py:179-197: strips cover every |Lambda| >= 1e-20 and no
    |Lambda| < 1e-50, with column cuts on multiples of 6 where possible."""
    lmax = 3 * nside
    nodes = osht.ring_thetas(nside, positive_only=True)
    L = osht.normalized_legendre(m, nodes, lmax, 1e-300).T
    mask = np.zeros(L.shape, bool)
    for rstart, rstop, cstart, cstop in stripify(L, include_above=1e-20, exclude_below=1e-50):
        assert cstart % 6 == 0 or L[0, cstart] == 0
        assert cstop == L.shape[1] or cstop % 6 == 0 or L[0, cstop] == 0
        mask[rstart:rstop, cstart:cstop] = True
    assert np.all(mask[np.abs(L) >= 1e-20])
    assert not np.any(mask[np.abs(L) < 1e-50])
