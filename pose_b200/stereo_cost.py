"""Fixed-point cost units and penalties: src/main/java/sgm/StereoCost.java:7-48, on the host.

These run once per call on the host, exactly as in the reference, and fill the ``csgm_params``
structure the C ABI takes.
"""
from __future__ import annotations

import math

from ._abi import CsgmParams

COST_CODES = {"census": 0, "ad-census": 1, "census-gradient": 2, "zncc": 3}


def java_round(v: float) -> int:
    """java.lang.Math.round(double): closest integer, ties toward positive infinity."""
    f = math.floor(v)
    return int(f + 1 if v - f >= 0.5 else f)


class StereoCost:
    @staticmethod
    def code(o) -> int:  # StereoCost.java:7-15
        try:
            return COST_CODES[o.matchingCost]
        except KeyError:
            raise ValueError("Unknown matching cost") from None

    @staticmethod
    def bits(o) -> int:
        return o.window_x * o.window_y - 1

    @staticmethod
    def penalty(value: float, o) -> int:  # StereoCost.java:17-19
        return java_round(value * StereoCost.bits(o) / 24.0)

    @staticmethod
    def p2(o) -> int:  # StereoCost.java:21-23
        return max(StereoCost.penalty(o.p1, o) + 1, StereoCost.penalty(o.p2, o))

    @staticmethod
    def aggregateBound(o) -> int:  # StereoCost.java:31-33
        return o.directions * (512 + StereoCost.p2(o))

    @staticmethod
    def aggregateBytes(o) -> int:  # StereoCost.java:35-41
        fits = StereoCost.aggregateBound(o) <= 65535
        if o.sgmAggregate == "16" and not fits:
            raise ValueError(
                "16-bit SGM aggregate cannot hold proved bound " + str(StereoCost.aggregateBound(o)))
        return 2 if o.sgmAggregate != "32" and fits else 4

    @staticmethod
    def pathP2(p1: int, p2: int, scale: int, gray, current: int, previous: int) -> int:
        """StereoCost.java:44-48."""
        if scale == 0:
            return p2
        difference = abs(int(gray[current]) - int(gray[previous]))
        return max(p1 + 1, (p2 * scale) // (scale + difference))


def params_from_options(o) -> CsgmParams:
    """The C-ABI parameter block for these options (the `costs`/`paths` kernel arguments,
    src/main/java/sgm/GpuStereo.java:384-403,600-614)."""
    p = CsgmParams()
    p.disparities = o.disparities
    p.min_disparity = o.minDisparity
    p.window_x = o.window_x
    p.window_y = o.window_y
    p.cost_mode = StereoCost.code(o)
    p.census_weight_milli = java_round(o.censusWeight * 1000)
    p.ad_truncation = o.adTruncation
    p.gradient_truncation = o.gradientTruncation
    p.p1 = StereoCost.penalty(o.p1, o)
    p.p2 = StereoCost.p2(o)
    p.edge_scale = o.sgmEdgeScale
    p.directions = o.directions
    p.aggregate_bytes = StereoCost.aggregateBytes(o)
    p.flags = 0
    p.uniqueness = float(o.uniqueness)
    p.lr_threshold = float(o.lrThreshold)
    return p
