"""Host-side checks of the C ABI (no GPU): the library loads, exports every
entry point declared in include/*.h, validates resource files and fails
cleanly on corrupt ones."""
import ctypes
import os
import re
import shutil
import struct

import numpy as np
import pytest

from wavemoth_b200 import _native
from wavemoth_b200 import lib as wlib

from .plans import plan_file

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in ("wavemoth.h", "wavemoth_b200.h"):
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b([a-z_][a-z0-9_]*)\s*\(", text):
            name = m.group(1)
            if name.startswith(("wavemoth_", "wm_", "bfm_")):
                names.add(name)
    return sorted(names)


def test_library_exports_every_declared_symbol():
    lib = _native.lib()
    names = declared_functions()
    assert len(names) >= 25
    for n in names:
        assert hasattr(lib, n), "missing export: " + n


def test_query_resourcefile():
    path = plan_file(4, 8, 4, 1e-10, 1.0)
    assert wlib.query_resourcefile(path) == (4, 8)
    with pytest.raises(IOError):
        wlib.query_resourcefile("/nonexistent/plan.dat")


def check(path, nside, lmax):
    st = (ctypes.c_int64 * 8)()
    rc = _native.lib().wavemoth_check_resourcefile(path.encode(), nside, lmax, st)
    return rc, wlib.last_error(), list(st)


@pytest.mark.parametrize("cfg", [(4, 8, 4, 1e-10, 1.0), (16, 32, 8, 1e-10, 1e-10),
                                 (32, 64, 16, 1e-10, 20.0)])
def test_check_resourcefile_accepts_writer_output(cfg):
    path = plan_file(*cfg)
    for _ in range(3):   # repeated compiles give the same program
        rc, err, st = check(path, cfg[0], cfg[1])
        assert rc == 0, err
    assert st[0] == 2 * (cfg[1] + 1)


def test_fault_injection_on_resource_files(tmp_path):
    """Truncated, corrupted and mismatched files fail with a message."""
    good = plan_file(16, 32, 8, 1e-10, 1e-10)
    data = open(good, "rb").read()
    cases = {}
    cases["truncated_header"] = data[:20]
    cases["truncated_body"] = data[: len(data) // 2]
    bad = bytearray(data)
    struct.pack_into("<q", bad, 24, len(data) + 1000)   # offset of m=0 even past EOF
    cases["offset_past_eof"] = bytes(bad)
    bad = bytearray(data)
    start = struct.unpack_from("<q", data, 24)[0]
    struct.pack_into("<i", bad, start + 4, 999)         # ncols of the first matrix
    cases["wrong_shape"] = bytes(bad)
    bad = bytearray(data)
    struct.pack_into("<q", bad, 24 + 8 * 2, 0)          # m=0 odd missing
    cases["missing_matrix"] = bytes(bad)
    for name, blob in cases.items():
        p = tmp_path / (name + ".dat")
        p.write_bytes(blob)
        rc, err, _ = check(str(p), 16, 32)
        assert rc == 2 and err, name
    p = tmp_path / "ok.dat"
    shutil.copy(good, p)
    rc, err, _ = check(str(p), 8, 32)
    assert rc == 2 and "Nside" in err
    rc, err, _ = check(str(p), 16, 30)
    assert rc == 2 and "lmax" in err


def test_random_byte_corruption_never_crashes(tmp_path):
    good = open(plan_file(8, 16, 8, 1e-10, 1.0), "rb").read()
    rng = np.random.default_rng(1)
    for i in range(60):
        bad = bytearray(good)
        for _ in range(8):
            bad[int(rng.integers(24, len(bad)))] = int(rng.integers(0, 256))
        p = tmp_path / ("c%d.dat" % i)
        p.write_bytes(bytes(bad))
        rc, err, _ = check(str(p), 8, 16)
        assert rc in (0, 2)


def test_plan_argument_validation():
    path = plan_file(4, 8, 4, 1e-10, 1.0)
    alm = np.zeros((45, 1), np.complex128)
    with pytest.raises(ValueError):
        wlib.ShtPlan(4, 8, 8, alm, np.zeros((191, 1)), "mmajor", matrix_data_filename=path)
    with pytest.raises(ValueError):
        wlib.ShtPlan(4, 8, 8, alm, np.zeros((192, 2)), "mmajor", matrix_data_filename=path)
    with pytest.raises(ValueError):
        wlib.ShtPlan(4, 8, 8, alm, np.zeros((192, 1)), "ringmajor", matrix_data_filename=path)
    L = _native.lib()
    assert not L.wavemoth_plan_to_healpix(4, 8, 7, 1, 1, None, None, 0, 0, path.encode())
    assert "mmax" in wlib.last_error()
    assert not L.wavemoth_plan_to_healpix(4, 8, 8, 1, 1, None, None, 0, 0, b"/nonexistent.dat")
    assert "cannot open" in wlib.last_error()


def test_no_gpu_plan_creation_fails_cleanly():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    path = plan_file(4, 8, 4, 1e-10, 1.0)
    with pytest.raises(wlib.WavemothError):
        wlib.ShtPlan(4, 8, 8, np.zeros((45, 1), np.complex128), np.zeros((192, 1)), "mmajor",
                     matrix_data_filename=path)


def test_interp_decomp_contract():
    rng = np.random.default_rng(0)
    A = rng.standard_normal((60, 8)) @ rng.standard_normal((8, 30))
    k, perm, proj = _native.interp_decomp(A, 1e-12)
    assert k == 8
    np.testing.assert_allclose(A[:, perm[k:]], A[:, perm[:k]] @ proj, atol=1e-9)
    k0, _, _ = _native.interp_decomp(np.zeros((5, 4)), 1e-10)
    assert k0 == 0


def test_every_declared_function_has_a_ctypes_signature():
    """Every C entry point of include/*.h is typed in wavemoth_b200._abi (or
    _native): an untyped ctypes call would pass 64-bit pointers as C ints."""
    from wavemoth_b200 import _abi, _native
    typed = set(_abi.SIGNATURES) | set(_native.HOST_SIGNATURES) | {"wavemoth_create_healpix_grid_info",
                                                                   "wavemoth_free_grid_info"}
    missing = [n for n in declared_functions() if n not in typed]
    assert not missing, missing
