"""Host interface of the B200 transform, mirroring the reference's Cython
layer (wavemoth/lib.pyx:113-218): ``ShtPlan`` with execute /
perform_legendre_transform / perform_backward_ffts / get_work, and
``_get_healpix_phi0s``.  Everything runs through the C ABI of
libwavemoth_b200.so; there is no CPU implementation behind it.
"""
import ctypes
import os

import numpy as np

from . import _native

WAVEMOTH_MMAJOR = 0x0
WAVEMOTH_ESTIMATE = 0x0
WAVEMOTH_MEASURE = 0x1
WAVEMOTH_NO_RESOURCE_COPY = 0x10
WAVEMOTH_DEVICE_POINTERS = 0x100
WAVEMOTH_PRECISION_SPLIT = 0x200
WAVEMOTH_SPLIT_GENERATE = 0x400
WAVEMOTH_DENSE = 0x800
# precision= of the plans: FP64 tensor cores, or the split int8 path with the
# residual P sliced once per plan ("split") or generated at every call
# ("split-generate", less device memory)
PRECISION_FLAGS = {"double": 0, "split": WAVEMOTH_PRECISION_SPLIT,
                   "split-generate": WAVEMOTH_PRECISION_SPLIT | WAVEMOTH_SPLIT_GENERATE}

_configured = False


class WavemothError(RuntimeError):
    pass


def _lib():
    return _native.lib()


def last_error():
    return _lib().wavemoth_last_error().decode(errors="replace")


def configure(resource_dir):
    """wavemoth_configure (src/wavemoth.h:33)."""
    global _configured
    _lib().wavemoth_configure(os.fsencode(resource_dir))
    _configured = True


def query_resourcefile(path):
    """(Nside, lmax), or raises if the file cannot be read (src/wavemoth.h:46)."""
    n, l = ctypes.c_int(), ctypes.c_int()
    rc = _lib().wavemoth_query_resourcefile(os.fsencode(path), ctypes.byref(n), ctypes.byref(l))
    if rc != 0:
        raise IOError("cannot read resource file header: %s" % path)
    return n.value, l.value


class ShtPlan:
    """alm2map plan (or map2alm with direction='map2alm').

    Arguments follow wavemoth/lib.pyx:118-152: input is the complex128 alm
    array (nalm, nmaps) in m-major order and output the float64 map
    (12 Nside^2, nmaps); for map2alm the roles are swapped.
    """

    def __init__(self, Nside, lmax, mmax, input, output, ordering, phase_shifts=True,
                 matrix_data_filename=None, nthreads=1, direction="alm2map", precision="double"):
        if ordering != "mmajor":
            raise ValueError("Invalid ordering: %s" % ordering)
        if direction not in ("alm2map", "map2alm"):
            raise ValueError("Invalid direction: %s" % direction)
        if precision not in PRECISION_FLAGS:
            raise ValueError("Invalid precision: %s" % precision)
        alm, maps = (input, output) if direction == "alm2map" else (output, input)
        if not (isinstance(alm, np.ndarray) and alm.dtype == np.complex128 and alm.ndim == 2
                and alm.flags.c_contiguous):
            raise ValueError("alm must be a C-contiguous complex128 (nalm, nmaps) array")
        if not (isinstance(maps, np.ndarray) and maps.dtype == np.float64 and maps.ndim == 2
                and maps.flags.c_contiguous):
            raise ValueError("map must be a C-contiguous float64 (npix, nmaps) array")
        if not (input.shape[1] == output.shape[1]):
            raise ValueError("Nonconforming arrays")
        if maps.shape[0] != 12 * Nside * Nside:
            raise ValueError("Output must have shape (Npix, nmaps), has %r" % (maps.shape,))
        if alm.shape[0] != (lmax + 1) * (lmax + 2) // 2:
            raise ValueError("alm must have (lmax+1)(lmax+2)/2 rows")
        if matrix_data_filename is None and not _configured:
            configure(os.environ["SHTRESOURCES"])
        self.input, self.output = input, output
        self.Nside, self.lmax, self.mmax = Nside, lmax, mmax
        self.nmaps = input.shape[1]
        self.direction = direction
        fn = (_lib().wavemoth_plan_to_healpix if direction == "alm2map"
              else _lib().wavemoth_plan_from_healpix)
        self._plan = fn(Nside, lmax, mmax, self.nmaps, nthreads,
                        input.ctypes.data, output.ctypes.data, WAVEMOTH_MMAJOR,
                        WAVEMOTH_ESTIMATE | PRECISION_FLAGS[precision],
                        None if matrix_data_filename is None else os.fsencode(matrix_data_filename))
        if not self._plan:
            raise WavemothError("Plan creation failed: " + last_error())
        if not phase_shifts:
            _lib().wavemoth_disable_phase_shifting(self._plan)

    def _check(self, what):
        st = _lib().wavemoth_plan_status(self._plan)
        if st != 0:
            raise WavemothError("%s failed (%d): %s" % (what, st, last_error()))

    def execute(self, repeat=1):
        for _ in range(repeat):
            _lib().wavemoth_execute(self._plan)
            self._check("execute")
        return self.output

    def execute_adjoint(self):
        """The adjoint of execute on the bound buffers: reads the output
        buffer, writes the input buffer (wavemoth_execute_adjoint)."""
        _lib().wavemoth_execute_adjoint(self._plan)
        self._check("execute_adjoint")
        return self.input

    def perform_legendre_transform(self, repeat=1):
        for _ in range(repeat):
            _lib().wavemoth_perform_legendre_transforms(self._plan)
            self._check("perform_legendre_transforms")

    def perform_backward_ffts(self):
        _lib().wavemoth_perform_backward_ffts(self._plan)
        self._check("perform_backward_ffts")

    def get_work(self):
        """complex128 (mmax+1, 2, 2 Nside, nmaps): the Legendre-phase output."""
        out = np.zeros((self.mmax + 1, 2, 2 * self.Nside, self.nmaps), np.complex128)
        rc = _lib().wavemoth_get_work(self._plan, out.view(np.float64).ctypes.data_as(
            ctypes.POINTER(ctypes.c_double)))
        if rc != 0:
            raise WavemothError("get_work failed: " + last_error())
        return out

    def legendre_flops(self, m, odd):
        return _lib().wavemoth_get_legendre_flops(self._plan, m, odd)

    @property
    def device_bytes(self):
        return _lib().wavemoth_plan_device_bytes(self._plan)

    @property
    def program_bytes(self):
        return _lib().wavemoth_plan_program_bytes(self._plan)

    def close(self):
        if getattr(self, "_plan", None):
            _lib().wavemoth_destroy_plan(self._plan)
            self._plan = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _get_healpix_phi0s(Nside):
    """phi0 of every ring from the C grid table (wavemoth/lib.pyx:203-213)."""
    info = _lib().wavemoth_create_healpix_grid_info(Nside)
    if not info:
        raise ValueError(last_error())
    try:
        g = info.contents
        return np.array([g.phi0s[i] for i in range(g.nrings)])
    finally:
        _lib().wavemoth_free_grid_info(info)


def get_healpix_grid(Nside):
    """(phi0s, ring_offsets, mid_ring, npix) from the C grid table."""
    info = _lib().wavemoth_create_healpix_grid_info(Nside)
    if not info:
        raise ValueError(last_error())
    try:
        g = info.contents
        phi0 = np.array([g.phi0s[i] for i in range(g.nrings)])
        offs = np.array([g.ring_offsets[i] for i in range(g.nrings + 1)], np.int64)
        return phi0, offs, g.mid_ring, g.npix
    finally:
        _lib().wavemoth_free_grid_info(info)
