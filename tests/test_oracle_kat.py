"""Pins the CPU oracle against the reference's own known-answer tests (CPU only).

Each test restates a check of the reference's regression suite on the same regenerated fixture.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

from fixtures import (plane_metrics, plane_pair, selftest_options, selftest_pair, shifted,
                      upgrade_pair)
from jrandom import JavaRandom
from pose_b200.options import Options
from pose_b200.stereo_cost import StereoCost, java_round
from reference_cpu import compute_cpu


def test_java_random_known_values():
    # Published values of the java.util.Random LCG.
    assert JavaRandom(42).nextInt() == -1170105035
    assert JavaRandom(0).nextInt() == -1155484576
    r = JavaRandom(42)
    assert [r.nextInt() for _ in range(3)] == [-1170105035, 234785527, -1360544799]


def test_java_round_ties(oracle_lib):
    for v, want in [(0.5, 1), (-0.5, 0), (2.5, 3), (-2.5, -2), (0.49999999999999994, 0),
                    (1e15 + 0.5, 1000000000000001)]:
        assert java_round(v) == want
        assert oracle_lib.java_round(v) == want


def test_penalty_units():
    """UpgradeStereoRegression.java:81-89."""
    c = Options()
    c.census = 5
    assert StereoCost.penalty(c.p1, c) == 4 and StereoCost.p2(c) == 24
    c.census = 11
    assert StereoCost.penalty(c.p1, c) == 20 and StereoCost.p2(c) == 120
    # 9x9 with p1=3, p2=36 gives the configs' effective P1=10, P2=120.
    c.census, c.p1, c.p2 = 9, 3, 36
    assert (StereoCost.penalty(c.p1, c), StereoCost.p2(c)) == (10, 120)
    assert StereoCost.aggregateBytes(c) == 2
    c.sgmAggregate = "32"
    assert StereoCost.aggregateBytes(c) == 4
    c.sgmAggregate, c.p2 = "16", 100000
    with pytest.raises(ValueError):
        StereoCost.aggregateBytes(c)


def test_selftest_sgm_known_answers(oracle_lib):
    """SelfTest.testSgm, SelfTest.java:81-114."""
    w, h, left, right = selftest_pair()
    o = selftest_options()
    d, _, _ = compute_cpu(o, left, right, w, h)
    region = d.reshape(h, w)[6:h - 6, 16:w - 8]
    finite = region[np.isfinite(region)]
    assert finite.size > 1500, "Textured stereo has enough consistent disparities"
    assert np.abs(finite - 6).mean() < 0.2, "Known 6-pixel disparity recovered"

    o.minDisparity, o.disparities = -10, 16
    rev, _, _ = compute_cpu(o, right, left, w, h)
    assert abs(rev[24 * w + 40] - (-6)) <= 0.3, "Signed disparity range"

    o.census, o.minDisparity, o.directions = 11, 0, 4
    d11, _, _ = compute_cpu(o, left, right, w, h)
    assert abs(d11[24 * w + 40] - 6) <= 0.3, "Multiword 11x11 census and four paths"

    constant = np.zeros(w * h, np.uint8)
    o.census = 5
    dc, _, _ = compute_cpu(o, constant, constant, w, h)
    assert math.isnan(dc[24 * w + 40]), "Ambiguous constant texture rejected"


@pytest.mark.parametrize("cost", ["census", "ad-census", "census-gradient", "zncc"])
@pytest.mark.parametrize("directions", [4, 8])
def test_upgrade_known_shift(oracle_lib, cost, directions):
    """UpgradeStereoRegression.java:35-54: known shift 13 and coverage for every cost."""
    w, h, shift, a, b, ma, mb = upgrade_pair()
    o = Options()
    o.disparities, o.minDisparity = 41, -3
    o.matchingCost, o.directions = cost, directions
    o.speckleSize, o.correlation, o.median = 0, 0.3, 1
    d, _, _ = compute_cpu(o, a, b, w, h, ma, mb)
    finite = d[np.isfinite(d)]
    good = int((np.abs(finite - shift) < 0.6).sum())
    assert finite.size > (w * h) // 2 and good > finite.size * 0.98


@pytest.mark.parametrize("cost", ["census", "ad-census", "census-gradient", "zncc"])
def test_matching_cost_plane(oracle_lib, cost):
    """MatchingCostBenchmark.java:17-34: >= 40000 valid and RMS <= 0.5 on the 13.37 px plane."""
    w, h, a, b = plane_pair()
    o = Options()
    o.disparities, o.median, o.speckleSize, o.correlation = 32, 1, 0, 0.5
    o.matchingCost = cost
    d, _, _ = compute_cpu(o, a, b, w, h)
    count, rms, _ = plane_metrics(d, w, h, 13.37)
    assert count >= 40000 and rms <= 0.5, (count, rms)


def test_census_bit_order(oracle_lib):
    """CensusSgm.census bit order: row-major window, centre skipped, bit k set iff neighbour < centre."""
    w, h = 7, 7
    img = np.arange(w * h, dtype=np.uint8)
    desc = oracle_lib.census(img, w, h, 3, 3)
    # centre (3,3)=24; neighbours in order: 16,17,18,23,25,30,31,32 -> first four are smaller
    assert int(desc[3 * w + 3]) == 0b00001111
    desc97 = oracle_lib.census(np.ascontiguousarray(JavaRandom(5).nextBytes(30 * 20)), 30, 20, 9, 7)
    assert desc97.size == 30 * 20 and int(desc97.max()) < (1 << 62)


def test_shifted_helper():
    a = np.arange(12, dtype=np.uint8)
    assert list(shifted(a, 4, 3, 1)) == [1, 2, 3, 3, 5, 6, 7, 7, 9, 10, 11, 11]
