"""CensusSgm.compute's host wiring, checked without a GPU.

A stand-in session routes the two device calls compute makes (the pair and the post-filters)
to the oracle, so the test exercises what runs on the host around them: the Options -> csgm_post
mapping (post_settings), the Stats round trip between the stages and the order of the stages.
The result must equal the oracle's computeRecorded (reference_cpu.compute_cpu) bit for bit.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

import oracle.oracle as orc
from pose_b200.options import Options
from pose_b200.sgm import CensusSgm, Result, Stats, post_settings
from pose_b200.synthetic import PairSpec, make_pair
from reference_cpu import compute_cpu, post_from_options


class OracleSession:
    """The GpuSgm calls CensusSgm.compute makes, answered by the oracle."""

    def set_streaming(self, mode="auto", strip_rows=64):
        self.streaming = (mode, strip_rows)

    def set_candidates(self, per_path=2):
        self.candidates = per_path

    def set_host_budget(self, nbytes=0):
        self.host_budget = nbytes

    def pair(self, params, left, right, w, h, validLeft=None, validRight=None, want_views=False,
             want_reasons=False, leftBgr=None, rightBgr=None):
        r = orc.pair(params, left, right, w, h, validLeft, validRight, want_reasons=True,
                     left_bgr=leftBgr, right_bgr=rightBgr)
        return Result(w, h, r["checked"], Stats.from_c(r["stats"]), r["dl"], r["dr"],
                      r["reasons"] if want_reasons else None,
                      r["boundary"] if want_reasons else None)

    def postfilter(self, post, left, right, disp_r, w, h, checked, reasons=None, stats=None,
                   leftBgr=None, rightBgr=None):
        opost = orc.OraclePost()
        ctypes.memmove(ctypes.byref(opost), ctypes.byref(post), ctypes.sizeof(opost))
        orc.postfilter(opost, left, right, disp_r, w, h, checked, stats, reasons,
                       left_bgr=leftBgr, right_bgr=rightBgr)
        return checked


def test_post_settings_match_the_oracle_mapping():
    o = Options()
    o.median, o.medianMode, o.speckleConnectivity, o.correlationWindow = 5, "classic", 4, 9
    a, b = post_settings(o), post_from_options(o)
    assert ctypes.sizeof(a) == ctypes.sizeof(b)
    assert ctypes.string_at(ctypes.addressof(a), ctypes.sizeof(a)) == \
        ctypes.string_at(ctypes.addressof(b), ctypes.sizeof(b))


def test_compute_equals_compute_recorded(oracle_lib):
    w, h = 160, 120
    left, right, _ = make_pair(PairSpec(w, h, planes=3, d_min=4, d_max=30, seed=21))
    o = Options()
    o.census, o.disparities = 9, 32
    want, want_stats, want_res = compute_cpu(o, left, right, w, h)
    got = CensusSgm(o, session=OracleSession()).compute(left, right, w, h, want_reasons=True)
    assert np.array_equal(got.disparity.view(np.uint32), want.view(np.uint32))
    assert np.array_equal(got.reasons, want_res["reasons"])
    for c_name, name in Stats._C_NAMES.items():
        assert getattr(got.stats, name) == getattr(want_stats, c_name), name


def test_color_mode_routes_bgr_images(oracle_lib):
    """--census-mode color-distance: CensusSgm.compute hands the BGR images to the pair and to
    the post-filters (CensusSgm.java:108-120,222-224) and refuses to run without them."""
    from pose_b200.synthetic import make_color_pair

    w, h = 64, 40
    left, right, lbgr, rbgr, _ = make_color_pair(PairSpec(w, h, planes=2, d_min=3, d_max=12,
                                                          seed=5))
    o = Options()
    o.census, o.disparities, o.censusMode = 5, 16, "color-distance"
    sgm = CensusSgm(o, session=OracleSession())
    with pytest.raises(ValueError):
        sgm.compute(left, right, w, h)
    got = sgm.compute(left, right, w, h, leftBgr=lbgr, rightBgr=rbgr)
    prm = sgm.params()
    want = orc.pair(prm, left, right, w, h, want_reasons=True, left_bgr=lbgr, right_bgr=rbgr)
    checked, st = want["checked"].copy(), want["stats"]
    post = orc.OraclePost()
    ctypes.memmove(ctypes.byref(post), ctypes.byref(post_settings(o)), ctypes.sizeof(post))
    orc.postfilter(post, left, right, want["dr"], w, h, checked, st, left_bgr=lbgr,
                   right_bgr=rbgr)
    assert np.array_equal(got.disparity.view(np.uint32), checked.view(np.uint32))
    assert got.stats.photometricRejected == st.photometric_rejected

