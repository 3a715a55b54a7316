"""Plan-file fixtures for the tests: rev1 files written by the package's
writer (wavemoth_b200.resource) into a per-session directory."""
import os
import tempfile

from wavemoth_b200 import resource

_DIR = None
_CACHE = {}


def plan_dir():
    global _DIR
    if _DIR is None:
        _DIR = tempfile.mkdtemp(prefix="wm_plans_")
    return _DIR


def plan_file(nside, lmax, chunk_size=64, eps=1e-10, memop_cost=20.0, workers=1):
    key = (nside, lmax, chunk_size, eps, memop_cost)
    if key not in _CACHE:
        path = os.path.join(plan_dir(), "plan_%d_%d_%d_%g_%g.dat" % key)
        rc = resource.ResourceComputer(nside, lmax, lmax, chunk_size, eps, memop_cost)
        with open(path, "wb") as f:
            rc.compute(f, max_workers=workers)
        _CACHE[key] = path
    return _CACHE[key]


def rel(a, b):
    import numpy as np
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))
