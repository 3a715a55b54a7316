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


def plan_file(nside, lmax, chunk_size=64, eps=1e-10, memop_cost=20.0, workers=1, max_levels=None):
    """Path of a plan file with these parameters, written on first use.  With
    WAVEMOTH_PLAN_DIR set, files are kept there under bench.py's names, so a
    test run and a bench run on one host write each large file once."""
    key = (nside, lmax, chunk_size, eps, memop_cost, max_levels)
    shared = os.environ.get("WAVEMOTH_PLAN_DIR")
    lv = "" if max_levels is None else "_levels%d" % max_levels
    if shared and key not in _CACHE:
        path = os.path.join(shared, "rev1_nside%d_lmax%d_eps%g_chunk%d_memop%g%s.dat"
                            % (nside, lmax, eps, chunk_size, memop_cost, lv))
        if not os.path.exists(path):
            os.makedirs(shared, exist_ok=True)
            resource.compute_resource_file(path, nside, lmax, chunk_size=chunk_size, eps=eps,
                                           memop_cost=memop_cost, max_workers=workers, max_levels=max_levels)
        _CACHE[key] = path
    if key not in _CACHE:
        path = os.path.join(plan_dir(), "plan_%d_%d_%d_%g_%g%s.dat" % (key[:5] + (lv,)))
        rc = resource.ResourceComputer(nside, lmax, lmax, chunk_size, eps, memop_cost, max_levels=max_levels)
        with open(path, "wb") as f:
            rc.compute(f, max_workers=workers)
        _CACHE[key] = path
    return _CACHE[key]


def rel(a, b):
    import numpy as np
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))
