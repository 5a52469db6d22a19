"""The C oracle (CPU loops of CensusSgm.match) and the numpy restatement of the reference's OpenCL
kernels must agree bit for bit, as the reference's CPU==GPU regressions require of its own two
implementations (StorageGpuRegression.java:68-90, ScalingRegression.java:56-99)."""
from __future__ import annotations

import numpy as np
import pytest

import kernel_restatement as kr
from fixtures import scaling_pair, storage_gpu_pair
from pose_b200.options import Options
from pose_b200.stereo_cost import params_from_options


def _views(orc, o, a, b, w, h, ma=None, mb=None):
    wx, wy = o.window_x, o.window_y
    da, db = orc.census(a, w, h, wx, wy), orc.census(b, w, h, wx, wy)
    ta, tb = orc.texture(a, w, h, wx, wy), orc.texture(b, w, h, wx, wy)
    if ma is not None:
        ta &= (ma != 0).astype(np.uint8)
        tb &= (mb != 0).astype(np.uint8)
    return da, db, ta, tb


@pytest.mark.parametrize("cost", ["census", "ad-census", "census-gradient", "zncc"])
@pytest.mark.parametrize("directions,bits", [(4, "16"), (8, "16"), (8, "32")])
@pytest.mark.parametrize("reverse", [0, 1])
def test_scaling_fixture_bit_exact(oracle_lib, cost, directions, bits, reverse):
    w, h, a, b, ma, mb = scaling_pair()
    o = Options()
    o.disparities, o.minDisparity = 33, -5
    o.matchingCost, o.directions, o.sgmAggregate = cost, directions, bits
    prm = params_from_options(o)
    da, db, ta, tb = _views(oracle_lib, o, a, b, w, h, ma, mb)
    if reverse:
        da, db, ta, tb, a, b = db, da, tb, ta, b, a
    ref = oracle_lib.match(prm, da, db, a, b, ta, tb, w, h, reverse, want_volumes=True,
                           want_summary=True)
    cost_k, S_k, summary_k, disp_k, st = kr.match(prm, da, db, a, b, ta, tb, w, h, reverse)
    assert np.array_equal(ref["cost"].astype(np.int64), cost_k.reshape(-1))
    assert np.array_equal(ref["aggregate"].astype(np.int64), S_k.reshape(-1))
    assert np.array_equal(ref["summary"].reshape(-1, 6).astype(np.int64), summary_k)
    assert np.array_equal(ref["disp"].view(np.uint32), disp_k.view(np.uint32))
    s = ref["stats"]
    assert (s.full_interval_pixels, s.boundary_rejected, s.lower_boundary_rejected,
            s.upper_boundary_rejected, s.ambiguity_rejected, s.selected) == (
        st["full"], st["boundary"], st["lower"], st["upper"], st["ambiguous"], st["selected"])


@pytest.mark.parametrize("census", [5, 11])
@pytest.mark.parametrize("directions", [4, 8])
def test_storage_fixture_bit_exact(oracle_lib, census, directions):
    w, h, a, b, mask = storage_gpu_pair()
    o = Options()
    o.census, o.directions = census, directions
    o.disparities = 177 if census == 11 else 37
    prm = params_from_options(o)
    da, db, ta, tb = _views(oracle_lib, o, a, b, w, h, mask, mask)
    ref = oracle_lib.match(prm, da, db, a, b, ta, tb, w, h, 0, want_summary=True)
    _, _, summary_k, disp_k, _ = kr.match(prm, da, db, a, b, ta, tb, w, h, 0)
    assert np.array_equal(ref["summary"].reshape(-1, 6).astype(np.int64), summary_k)
    assert np.array_equal(ref["disp"].view(np.uint32), disp_k.view(np.uint32))


def test_rectangular_window_and_no_edge_scale(oracle_lib):
    """Extension pin: 9x7 census (one word) and sgmEdgeScale 0 through both restatements."""
    w, h, a, b, ma, mb = scaling_pair()
    o = Options()
    o.census, o.censusHeight, o.disparities, o.sgmEdgeScale = 9, 7, 24, 0
    prm = params_from_options(o)
    da, db, ta, tb = _views(oracle_lib, o, a, b, w, h, ma, mb)
    ref = oracle_lib.match(prm, da, db, a, b, ta, tb, w, h, 0, want_volumes=True,
                           want_summary=True)
    cost_k, S_k, summary_k, disp_k, _ = kr.match(prm, da, db, a, b, ta, tb, w, h, 0)
    assert np.array_equal(ref["aggregate"].astype(np.int64), S_k.reshape(-1))
    assert np.array_equal(ref["disp"].view(np.uint32), disp_k.view(np.uint32))
