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


POST_CASES = {
    "defaults": {},
    "classic_5": {"median": 5, "medianMode": "classic"},
    "edge_7_no_gray_gate": {"median": 7, "medianEdgeThreshold": 0, "medianMaxChange": 0.25},
    "tight_gate_9": {"median": 1, "correlation": 0.9, "correlationWindow": 9},
    "four_connected": {"speckleConnectivity": 4, "speckleSize": 30, "speckleRange": 0.5},
}


@pytest.mark.parametrize("case", sorted(POST_CASES))
def test_postfilter_restatement_bit_exact(oracle_lib, case):
    """The C oracle's post-filters equal the independent Python restatement of
    CensusSgm.java:203-272 bit for bit (map, reasons, counters)."""
    import postfilter_restatement as pr
    from pose_b200.synthetic import PairSpec, make_pair
    from reference_cpu import post_from_options

    orc = oracle_lib
    w, h = 72, 54
    left, right, _ = make_pair(PairSpec(w, h, planes=3, d_min=3, d_max=14, seed=7))
    o = Options()
    o.census, o.disparities = 5, 16
    for k, v in POST_CASES[case].items():
        setattr(o, k, v)
    res = orc.pair(params_from_options(o), left, right, w, h, want_reasons=True)
    post = post_from_options(o)

    want = res["checked"].copy()
    want_reasons = res["reasons"].copy()
    stats = res["stats"]
    base = {k: getattr(stats, k) for k in ("post_median_lr_rejected", "photometric_rejected",
                                           "valid")}
    orc.postfilter(post, left, right, res["dr"], w, h, want, stats, want_reasons)

    mine = res["checked"].copy()
    mine_reasons = res["reasons"].copy()
    counts = {"postMedianLrRejected": base["post_median_lr_rejected"],
              "photometricRejected": base["photometric_rejected"], "speckleRejected": 0,
              "valid": base["valid"]}
    settings = {"median": o.median, "classic": o.medianMode == "classic",
                "max_change": o.medianMaxChange, "edge": o.medianEdgeThreshold,
                "lr": o.lrThreshold, "border": o.census // 2, "window": o.correlationWindow,
                "correlation": o.correlation, "speckle": o.speckleSize, "range": o.speckleRange,
                "connectivity": o.speckleConnectivity}
    pr.postfilter(settings, left, right, res["dr"], w, h, mine, counts, mine_reasons)

    assert np.array_equal(mine.view(np.uint32), want.view(np.uint32)), case
    assert np.array_equal(mine_reasons, want_reasons), case
    assert counts["postMedianLrRejected"] == stats.post_median_lr_rejected
    assert counts["photometricRejected"] == stats.photometric_rejected
    assert counts["speckleRejected"] == stats.speckle_rejected
    assert counts["valid"] == stats.valid
    assert (np.isfinite(res["checked"]) & ~np.isfinite(want)).any(), case


@pytest.mark.parametrize("case", ["edge", "classic", "gate_off"])
def test_color_postfilter_restatement_bit_exact(oracle_lib, case):
    """--census-mode color-distance: the oracle's post-filters with the three-channel photometric
    gate on the BGR images (CensusSgm.java:222-224,240-250) equal the restatement bit for bit,
    on the oracle's own colour-census pair."""
    import postfilter_restatement as pr
    from pose_b200.synthetic import PairSpec, make_color_pair
    from reference_cpu import post_from_options

    orc = oracle_lib
    w, h = 72, 54
    left, right, lbgr, rbgr, _ = make_color_pair(PairSpec(w, h, planes=3, d_min=3, d_max=14,
                                                          seed=17))
    o = Options()
    o.census, o.disparities = 5, 16
    o.correlation = 0.55 if case != "gate_off" else -1.0
    if case == "classic":
        o.medianMode = "classic"
    res = orc.pair(params_from_options(o), left, right, w, h, want_reasons=True, left_bgr=lbgr,
                   right_bgr=rbgr)
    post = post_from_options(o)
    want, want_reasons, stats = res["checked"].copy(), res["reasons"].copy(), res["stats"]
    base = (stats.post_median_lr_rejected, stats.photometric_rejected, stats.valid)
    orc.postfilter(post, left, right, res["dr"], w, h, want, stats, want_reasons,
                   left_bgr=lbgr, right_bgr=rbgr)
    mine, mine_reasons = res["checked"].copy(), res["reasons"].copy()
    counts = {"postMedianLrRejected": base[0], "photometricRejected": base[1],
              "speckleRejected": 0, "valid": base[2]}
    settings = {"median": o.median, "classic": o.medianMode == "classic",
                "max_change": o.medianMaxChange, "edge": o.medianEdgeThreshold,
                "lr": o.lrThreshold, "border": o.census // 2, "window": o.correlationWindow,
                "correlation": o.correlation, "speckle": o.speckleSize, "range": o.speckleRange,
                "connectivity": o.speckleConnectivity}
    pr.postfilter(settings, left, right, res["dr"], w, h, mine, counts, mine_reasons,
                  left_bgr=lbgr, right_bgr=rbgr)
    assert np.array_equal(mine.view(np.uint32), want.view(np.uint32)), case
    assert np.array_equal(mine_reasons, want_reasons), case
    assert counts["photometricRejected"] == stats.photometric_rejected
    assert counts["valid"] == stats.valid
    if case != "gate_off":
        assert stats.photometric_rejected > base[1], "the colour gate rejected nothing"


def test_color_pair_is_the_composition(oracle_lib):
    """oracle_pair_color = colour census of both images + CensusSgm.match of both views + LR."""
    from pose_b200.synthetic import PairSpec, make_color_pair

    orc = oracle_lib
    w, h = 64, 40
    left, right, lbgr, rbgr, _ = make_color_pair(PairSpec(w, h, planes=2, d_min=3, d_max=12,
                                                          seed=5))
    o = Options()
    o.census, o.disparities = 5, 16
    prm = params_from_options(o)
    res = orc.pair(prm, left, right, w, h, want_reasons=True, left_bgr=lbgr, right_bgr=rbgr)
    da, ta = orc.color_census(lbgr, w, h, 5, 5)
    db, tb = orc.color_census(rbgr, w, h, 5, 5)
    dl = orc.match(prm, da, db, left, right, ta, tb, w, h, 0)["disp"]
    dr = orc.match(prm, db, da, right, left, tb, ta, w, h, 1)["disp"]
    checked, _ = orc.lr_check(dl, dr, w, h, 2, 2, prm.lr_threshold)
    assert np.array_equal(res["dl"].view(np.uint32), dl.view(np.uint32))
    assert np.array_equal(res["dr"].view(np.uint32), dr.view(np.uint32))
    assert np.array_equal(res["checked"].view(np.uint32), checked.view(np.uint32))
    gray = orc.pair(prm, left, right, w, h)
    assert not np.array_equal(gray["dl"].view(np.uint32), dl.view(np.uint32))


@pytest.mark.parametrize("wx,wy", [(3, 3), (5, 5), (9, 7), (11, 11)])
def test_color_census_restatement_bit_exact(oracle_lib, wx, wy):
    """oracle_color_census equals the Python restatement of CensusSgm.colorCensus."""
    import postfilter_restatement as pr

    rng = np.random.default_rng(wx * 31 + wy)
    w, h = 37, 29
    bgr = rng.integers(0, 256, (h, w, 3)).astype(np.uint8)
    bgr[5:15, 5:20] = (40, 80, 120)  # an untextured patch
    want_desc, want_tex = oracle_lib.color_census(bgr.reshape(-1), w, h, wx, wy)
    desc, tex = pr.color_census(bgr.reshape(-1), w, h, wx, wy)
    assert np.array_equal(np.asarray(want_desc).reshape(-1), desc.reshape(-1))
    assert np.array_equal(np.asarray(want_tex).astype(bool), tex)
    assert tex.any() and not tex.all()
