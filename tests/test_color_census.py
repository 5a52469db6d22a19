"""GPU colour-distance census (csgm_color_census) against the oracle's restatement of
CensusSgm.colorCensus (CensusSgm.java:302-332): descriptors and texture bit for bit."""
from __future__ import annotations

import numpy as np
import pytest

import oracle.oracle as orc

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def session():
    from pose_b200.sgm import GpuSgm

    s = GpuSgm(0)
    yield s
    s.close()


def bgr_image(w, h, seed):
    """Smooth colour ramps with noise, a flat patch (untextured) and a hard edge."""
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:h, 0:w]
    img = np.stack([(xx * 3 + yy) % 256, (yy * 5) % 256, (xx * yy) % 256], -1).astype(np.int32)
    img += rng.integers(-6, 7, img.shape)
    img[h // 4:h // 2, w // 4:w // 2] = (90, 120, 150)
    img[:, (3 * w) // 4:] = 255 - img[:, (3 * w) // 4:]
    return np.clip(img, 0, 255).astype(np.uint8).reshape(-1)


@pytest.mark.parametrize("w,h,seed", [(64, 48, 1), (101, 37, 2)])
@pytest.mark.parametrize("wx,wy", [(3, 3), (5, 5), (9, 7), (9, 9), (11, 11)])
def test_color_census_matches_oracle(session, w, h, seed, wx, wy):
    bgr = bgr_image(w, h, seed)
    want_desc, want_tex = orc.color_census(bgr, w, h, wx, wy)
    desc, tex = session.color_census(bgr, w, h, wx, wy)
    assert np.array_equal(desc.reshape(-1), np.asarray(want_desc).reshape(-1))
    assert np.array_equal(tex.astype(bool), np.asarray(want_tex).astype(bool))
    assert tex.any() and not tex.all()


def color_pair(w=160, h=96, seed=31):
    from pose_b200.synthetic import PairSpec, make_color_pair

    return make_color_pair(PairSpec(w, h, planes=3, d_min=4, d_max=30, seed=seed))


@pytest.mark.parametrize("cost,directions,wx", [("census", 8, 5), ("census", 4, 9),
                                                ("ad-census", 8, 7), ("census-gradient", 16, 5),
                                                ("zncc", 8, 7)])
def test_pair_color_equals_oracle(session, cost, directions, wx):
    """csgm_pair_color (--census-mode color-distance, CensusSgm.java:108-201): colour-census
    descriptors and texture of the BGR images, gray costs and penalties, both views and the LR
    check, masks on both sides, on the fused and the general kernels, against the oracle."""
    from pose_b200.options import Options
    from pose_b200.stereo_cost import params_from_options

    left, right, lbgr, rbgr, _ = color_pair()
    w, h = 160, 96
    ma = np.full(w * h, 255, np.uint8)
    ma[20 * w:30 * w] = 0
    mb = np.full(w * h, 255, np.uint8)
    o = Options()
    o.census, o.disparities, o.matchingCost, o.directions = wx, 40, cost, directions
    prm = params_from_options(o)
    want = orc.pair(prm, left, right, w, h, ma, mb, want_reasons=True, left_bgr=lbgr,
                    right_bgr=rbgr)
    for flags in (0, 1):
        prm.flags = flags
        got = session.pair(prm, left, right, w, h, ma, mb, want_views=True, want_reasons=True,
                           leftBgr=lbgr, rightBgr=rbgr)
        assert np.array_equal(got.left.view(np.uint32), want["dl"].view(np.uint32))
        assert np.array_equal(got.right.view(np.uint32), want["dr"].view(np.uint32))
        assert np.array_equal(got.disparity.view(np.uint32), want["checked"].view(np.uint32))
        assert np.array_equal(got.reasons, want["reasons"])
        assert np.array_equal(got.searchBoundary, want["boundary"])
    if cost != "zncc":  # ZNCC reads the gray windows, not the descriptors
        gray = orc.pair(prm, left, right, w, h, ma, mb)
        assert not np.array_equal(gray["dl"].view(np.uint32), want["dl"].view(np.uint32))


@pytest.mark.parametrize("median_mode", ["edge-preserving", "classic"])
def test_compute_color_mode_equals_oracle(session, median_mode):
    """CensusSgm.compute in colour-distance mode: the pair from colour descriptors, then the
    post-filters with the three-channel photometric gate (CensusSgm.java:222-224,240-250)."""
    from pose_b200.options import Options
    from pose_b200.sgm import CensusSgm, post_settings

    left, right, lbgr, rbgr, _ = color_pair(seed=41)
    w, h = 160, 96
    o = Options()
    o.census, o.disparities, o.censusMode, o.medianMode = 5, 40, "color-distance", median_mode
    sgm = CensusSgm(o, session=session)
    got = sgm.compute(left, right, w, h, want_reasons=True, leftBgr=lbgr, rightBgr=rbgr)
    prm = sgm.params()
    want = orc.pair(prm, left, right, w, h, want_reasons=True, left_bgr=lbgr, right_bgr=rbgr)
    checked, reasons, st = want["checked"].copy(), want["reasons"].copy(), want["stats"]
    post = orc.OraclePost()
    import ctypes

    ctypes.memmove(ctypes.byref(post), ctypes.byref(post_settings(o)), ctypes.sizeof(post))
    orc.postfilter(post, left, right, want["dr"], w, h, checked, st, reasons, left_bgr=lbgr,
                   right_bgr=rbgr)
    assert np.array_equal(got.disparity.view(np.uint32), checked.view(np.uint32))
    assert np.array_equal(got.reasons, reasons)
    assert (got.stats.postMedianLrRejected, got.stats.photometricRejected,
            got.stats.speckleRejected, got.stats.valid) == (
        st.post_median_lr_rejected, st.photometric_rejected, st.speckle_rejected, st.valid)
    assert st.photometric_rejected > 0
