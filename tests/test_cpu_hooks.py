"""Host-side kernel-level hooks against the reference's own C library
(oracle/_ref): the packing of the SSE Legendre transform, the recurrence
coefficients, the work-size query, the matrix-header reader and the
butterfly scatter (src/legendre_transform.c.in:330-380, 625-633, 723-747;
src/butterfly.c.in:57-139, 434-445).  Bit-for-bit equality throughout."""
import ctypes
import io

import numpy as np
import pytest

from wavemoth_b200 import _native
from wavemoth_b200.resource import ArrayProvider, butterfly_compress, serialize_butterfly_matrix

from . import hooks_util as H


@pytest.fixture(scope="module")
def libs():
    from oracle import ref
    if not ref.available():
        pytest.skip("reference C library not available")
    return H.declare_hooks(_native.lib()), H.declare_hooks(ref.lib())


@pytest.mark.parametrize("nvecs", [2, 4, 6, 10, 12, 22])
@pytest.mark.parametrize("nk", [2, 3, 10, 42, 43, 44, 90])
def test_pack_matches_reference(libs, nk, nvecs):
    ours, ref = libs
    abig = np.random.default_rng(nk * 100 + nvecs).standard_normal((2 * nk, nvecs))
    assert np.array_equal(H.pack(ours, abig, nk), H.pack(ref, abig, nk))


@pytest.mark.parametrize("m,lmin,nk", [(0, 0, 3), (10, 210, 11), (3, 5, 40), (500, 500, 300), (2047, 2047, 2)])
def test_auxdata_matches_reference(libs, m, lmin, nk):
    ours, ref = libs
    assert np.array_equal(H.auxdata(ours, m, lmin, nk), H.auxdata(ref, m, lmin, nk))


@pytest.mark.parametrize("nvecs", [2, 4, 6, 64, 200])
def test_sse_query_work_matches_reference(libs, nvecs):
    ours, ref = libs
    assert ours.wavemoth_legendre_transform_sse_query_work(nvecs) == \
        ref.wavemoth_legendre_transform_sse_query_work(nvecs)


def test_query_matrix_data():
    lib = _native.lib()
    i, j = np.ogrid[:20, :10]
    A = (i * j).astype(np.float64)
    data = serialize_butterfly_matrix(butterfly_compress(A, chunk_size=3), ArrayProvider(A),
                                      num_levels=2).getvalue()
    buf = ctypes.create_string_buffer(data, len(data))

    class Info(ctypes.Structure):
        _fields_ = [(n, ctypes.c_size_t) for n in ("nrows", "ncols", "k_max", "nblocks_max", "element_count",
                                                     "first_level_size", "heap_size", "heap_first_index")]
    info = Info()
    end = lib.bfm_query_matrix_data(ctypes.addressof(buf), ctypes.addressof(info))
    assert end - ctypes.addressof(buf) == 40
    assert (info.nrows, info.ncols) == (20, 10)
    import struct
    h = struct.unpack_from("<iiiiqiiii", data, 0)
    assert (info.k_max, info.nblocks_max, info.element_count) == (h[2], h[3], h[4])
    assert (info.first_level_size, info.heap_size, info.heap_first_index) == (h[5], h[6], h[7])


@pytest.mark.parametrize("group", [0, 1])
@pytest.mark.parametrize("should_add", [0, 1])
@pytest.mark.parametrize("nvecs", [2, 6])
def test_scatter_matches_reference(libs, group, should_add, nvecs):
    ours, ref = libs
    rng = np.random.default_rng(7 + group + 2 * should_add + nvecs)
    len1, len2 = 13, 9
    mask = rng.integers(0, 2, len1 + len2)
    src = rng.standard_normal((int((mask == group).sum()) + 1, nvecs))
    out = []
    for L in (ours, ref):
        t1 = np.full((len1, nvecs), 0.5)
        t2 = np.full((len2, nvecs), -0.25)
        used = H.scatter(L, mask, t1, t2, src, group, should_add)
        out.append((used, t1, t2))
    assert out[0][0] == out[1][0] == len1 + len2
    assert np.array_equal(out[0][1], out[1][1]) and np.array_equal(out[0][2], out[1][2])
