"""The plan-file writer's depth cap (ResourceComputer(max_levels=...)).

The level choice of every matrix follows the writer's cost model
(wavemoth/lib.pyx:518-543) over the levels 0..min(depth, max_levels).  With
a tiny memop_cost the model asks for deep trees at nside 128, so the capped
file must hold fewer interpolation levels than the uncapped one, and at
most one per matrix."""
import ctypes
import os

from wavemoth_b200 import _native, resource

from .plans import plan_file


def _stats(path, nside, lmax):
    st = (ctypes.c_int64 * 8)()
    rc = _native.lib().wavemoth_check_resourcefile(os.fsencode(path), nside, lmax, st)
    assert rc == 0
    return list(st)


def test_max_levels_caps_every_matrix():
    nside, lmax = 128, 256
    free = plan_file(nside, lmax, 64, 1e-10, 1e-10, workers=4)
    capped = plan_file(nside, lmax, 64, 1e-10, 1e-10, workers=4, max_levels=1)
    s_free, s_cap = _stats(free, nside, lmax), _stats(capped, nside, lmax)
    nmats, levels = s_cap[0], s_cap[3]
    assert s_free[0] == nmats
    assert levels <= nmats
    assert s_free[3] > levels  # the cost model chose depth 2 somewhere without the cap


def test_max_levels_zero_writes_dense_residuals():
    rc = resource.ResourceComputer(64, 128, 128, memop_cost=1e-10, max_levels=0)
    assert rc.max_levels == 0


def test_max_levels_rejects_negative():
    import pytest
    with pytest.raises(ValueError):
        resource.ResourceComputer(16, 32, 32, max_levels=-1)
