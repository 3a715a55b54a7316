"""B200-native implementation of Wavemoth's spherical harmonic transform
(alm2map / map2alm on HEALPix grids with butterfly-compressed Legendre
matrices).  The compute path is libwavemoth_b200.so (CUDA, sm_100a) behind
the C ABI in include/wavemoth.h and include/wavemoth_b200.h."""
from . import healpix  # noqa: F401
from .lib import ShtPlan, configure, query_resourcefile, WavemothError  # noqa: F401
