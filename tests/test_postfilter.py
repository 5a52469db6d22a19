"""GPU post-filters (csgm_postfilter) against the oracle's restatement of
CensusSgm.computeRecorded :203-272 (median, post-median reciprocity, ZNCC photometric gate,
speckle removal, counters and reason codes), bit for bit.

The inputs are the GPU matcher's own outputs (LR-checked map, right view, reasons, counters),
which the parity tests pin to the oracle; both post-filters start from copies of them.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

import oracle.oracle as orc
from pose_b200 import _abi
from pose_b200.options import Options
from pose_b200.stereo_cost import params_from_options
from pose_b200.synthetic import PairSpec, make_pair
from reference_cpu import post_from_options

pytestmark = pytest.mark.gpu

CASES = {
    "defaults": {},
    "classic_median_5": {"median": 5, "medianMode": "classic"},
    "edge_median_11_no_gray_gate": {"median": 11, "medianEdgeThreshold": 0,
                                    "medianMaxChange": 0.25},
    "no_median_tight_gate": {"median": 1, "correlation": 0.9, "correlationWindow": 15},
    "four_connected_large_speckles": {"speckleConnectivity": 4, "speckleSize": 400,
                                      "speckleRange": 0.5},
    "no_speckles_no_gate": {"speckleSize": 0, "correlation": -1.0, "median": 7},
    "small_window_strict_lr": {"correlationWindow": 3, "lrThreshold": 0.25, "speckleSize": 1},
}


@pytest.fixture(scope="module")
def session():
    from pose_b200.sgm import GpuSgm

    s = GpuSgm(0)
    yield s
    s.close()


@pytest.fixture(scope="module", params=[(320, 240, 5), (301, 177, 9)], ids=["320x240", "301x177"])
def matched(request, session):
    w, h, seed = request.param
    left, right, _ = make_pair(PairSpec(w, h, planes=3, d_min=4, d_max=40, seed=seed))
    o = Options()
    o.census, o.disparities = 9, 64
    got = session.pair(params_from_options(o), left, right, w, h, want_views=True,
                       want_reasons=True)
    return w, h, left, right, got


def copy_stats(s):
    out = _abi.CsgmStats()
    ctypes.memmove(ctypes.byref(out), ctypes.byref(s), ctypes.sizeof(out))
    return out


@pytest.mark.parametrize("case", sorted(CASES))
def test_postfilter_matches_oracle(session, matched, case):
    w, h, left, right, got = matched
    o = Options()
    o.census, o.disparities = 9, 64
    for k, v in CASES[case].items():
        setattr(o, k, v)
    opost = post_from_options(o)
    post = _abi.CsgmPost()
    ctypes.memmove(ctypes.byref(post), ctypes.byref(opost), ctypes.sizeof(post))
    base_stats = got.stats.to_c()

    want = got.disparity.copy()
    want_reasons = got.reasons.copy()
    want_stats = copy_stats(base_stats)
    orc.postfilter(opost, left, right, got.right, w, h, want, want_stats, want_reasons)

    mine = got.disparity.copy()
    mine_reasons = got.reasons.copy()
    mine_stats = copy_stats(base_stats)
    session.postfilter(post, left, right, got.right, w, h, mine, mine_reasons, mine_stats)

    assert np.array_equal(mine.view(np.uint32), want.view(np.uint32)), case
    assert np.array_equal(mine_reasons, want_reasons), case
    for name in _abi.STATS_FIELDS:
        assert getattr(mine_stats, name) == getattr(want_stats, name), (case, name)
    # The filters did something in every case but the one that switches them off.
    if case != "no_speckles_no_gate":
        assert (np.isfinite(got.disparity) & ~np.isfinite(mine)).any(), case


def test_postfilter_twice_is_repeatable(session, matched):
    w, h, left, right, got = matched
    o = Options()
    o.census = 9
    post = _abi.CsgmPost()
    ctypes.memmove(ctypes.byref(post), ctypes.byref(post_from_options(o)), ctypes.sizeof(post))
    a = got.disparity.copy()
    b = got.disparity.copy()
    session.postfilter(post, left, right, got.right, w, h, a)
    session.postfilter(post, left, right, got.right, w, h, b)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
