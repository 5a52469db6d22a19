"""``new CensusSgm(o).compute(...)`` with compute=cpu, expressed through the C oracle.

This is what the reference's regressions call "expected" (the CPU side of every CPU==GPU check):
oracle_pair (CensusSgm.java:56-201) followed by oracle_postfilter (CensusSgm.java:203-272).
"""
from __future__ import annotations

import numpy as np

import oracle.oracle as orc
from pose_b200.stereo_cost import params_from_options


def post_from_options(o) -> "orc.OraclePost":
    post = orc.OraclePost()
    post.median = o.median
    post.median_classic = 1 if o.medianMode == "classic" else 0
    post.median_edge_threshold = o.medianEdgeThreshold
    post.correlation_window = o.correlationWindow
    post.speckle_size = o.speckleSize
    post.speckle_connectivity = o.speckleConnectivity
    post.border = o.census // 2
    post.median_max_change = o.medianMaxChange
    post.correlation = o.correlation
    post.lr_threshold = o.lrThreshold
    post.speckle_range = o.speckleRange
    return post


def compute_cpu(o, left, right, w, h, valid_l=None, valid_r=None, with_post=True):
    """Returns (disparity float32[n], stats CsgmStats, pair-dict)."""
    prm = params_from_options(o)
    res = orc.pair(prm, left, right, w, h, valid_l, valid_r, want_reasons=True)
    disp = res["checked"].copy()
    stats = res["stats"]
    if with_post:
        orc.postfilter(post_from_options(o), left, right, res["dr"], w, h, disp, stats,
                       res["reasons"])
    return disp, stats, res


def stats_csv(stats) -> str:
    """CensusSgm.Stats.csv (CensusSgm.java:718-736)."""
    return ",".join(str(getattr(stats, k)) for k in (
        "boundary_rejected", "upper_boundary_rejected", "ambiguity_rejected", "selected",
        "lr_rejected", "post_median_lr_rejected", "photometric_rejected", "speckle_rejected",
        "valid"))


def finite_count(d: np.ndarray) -> int:
    return int(np.isfinite(d).sum())


def compute_recorded_cpu(o, a, b, ca, cb, w, h, ma, mb):
    """CensusSgm.computeRecorded with compute=cpu and a collecting observer, as the pyramid
    matcher's tiles call it (DenseMatcher.java:306-318): a Result with reasons and flags."""
    from pose_b200.sgm import Result, Stats

    prm = params_from_options(o)
    res = orc.pair(prm, a, b, w, h, ma, mb, want_reasons=True, left_bgr=ca, right_bgr=cb)
    disp, stats, reasons = res["checked"].copy(), res["stats"], res["reasons"].copy()
    orc.postfilter(post_from_options(o), a, b, res["dr"], w, h, disp, stats, reasons,
                   left_bgr=ca, right_bgr=cb)
    return Result(w, h, disp, Stats.from_c(stats), res["dl"], res["dr"], reasons,
                  res["boundary"])

