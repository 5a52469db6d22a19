"""Streamed views (--gpu-sgm streamed / auto over budget): strips of rows with path-state carries,
the partial aggregate parked in pinned host memory between a down pass and an up pass
(GpuStereo.java:339-437 and the plan of :33-84).  Every streamed result is compared with the
oracle bit for bit and with the resident run on the same inputs, with at least three strips.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle.oracle as orc
from fixtures import scaling_pair, upgrade_pair
from pose_b200 import _abi
from pose_b200.options import Options
from pose_b200.stereo_cost import params_from_options

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def stats_tuple(s):
    return tuple(int(getattr(s, k)) for k in _abi.STATS_FIELDS)


def assert_same(got, want, what):
    assert np.array_equal(bits(got.left), bits(want["dl"])), f"{what}: left view"
    assert np.array_equal(bits(got.right), bits(want["dr"])), f"{what}: right view"
    assert np.array_equal(bits(got.disparity), bits(want["checked"])), f"{what}: LR-checked"
    assert np.array_equal(got.reasons, want["reasons"]), f"{what}: reasons"
    assert np.array_equal(got.searchBoundary, want["boundary"]), f"{what}: boundary flags"
    assert stats_tuple(got.stats.to_c()) == stats_tuple(want["stats"]), f"{what}: counters"


@pytest.fixture(scope="module")
def session():
    from pose_b200.sgm import GpuSgm

    orc.set_threads(8)
    s = GpuSgm(0)
    yield s
    s.close()


@pytest.mark.parametrize("cost", ["census", "ad-census", "zncc"])
@pytest.mark.parametrize("directions,agg", [(4, "16"), (8, "16"), (8, "32"), (16, "16"),
                                            (16, "32")])
def test_forced_streaming_equals_oracle(session, cost, directions, agg):
    """UpgradeStereoRegression's masked fixture (192x79, D41, minD -3) in strips of 16 rows."""
    w, h, _, a, b, ma, mb = upgrade_pair()
    o = Options()
    o.disparities, o.minDisparity = 41, -3
    o.matchingCost, o.directions, o.sgmAggregate = cost, directions, agg
    prm = params_from_options(o)
    want = orc.pair(prm, a, b, w, h, ma, mb, want_reasons=True)
    session.set_streaming("streamed", 16)
    try:
        plan = session.plan_detail(prm, w, h)
        assert plan["streamed"] and plan["rows"] == 16 and (h + 15) // 16 >= 3
        assert plan["host_bytes"] == w * h * o.disparities * prm.aggregate_bytes
        got = session.pair(prm, a, b, w, h, ma, mb, want_views=True, want_reasons=True)
    finally:
        session.set_streaming("auto")
    assert_same(got, want, f"streamed {cost} {directions}-path uint{8 * prm.aggregate_bytes}")


@pytest.mark.parametrize("rows", [1, 2, 3, 7])
def test_strip_heights(session, rows):
    """Strips down to one row (two with 16 paths), uneven last strips, against the oracle."""
    w, h, a, b, ma, mb = scaling_pair()
    for directions in (8, 16):
        o = Options()
        o.disparities, o.minDisparity, o.directions = 33, -5, directions
        prm = params_from_options(o)
        want = orc.pair(prm, a, b, w, h, ma, mb, want_reasons=True)
        session.set_streaming("streamed", rows)
        try:
            plan = session.plan_detail(prm, w, h)
            assert plan["rows"] == (max(rows, 2) if directions == 16 else rows)
            got = session.pair(prm, a, b, w, h, ma, mb, want_views=True, want_reasons=True)
        finally:
            session.set_streaming("auto")
        assert_same(got, want, f"{directions}-path strips of {plan['rows']} rows")


def test_auto_streams_when_the_budget_is_short():
    """A budget below the resident plan: auto mode streams (at least three strips), resident mode
    refuses before any work, and the streamed pair equals the resident one and the oracle."""
    from pose_b200.sgm import GpuSgm
    from pose_b200.synthetic import make_pair, spec_for

    left, right, _ = make_pair(spec_for("cfg1"))
    w, h, y0 = 1600, 200, 400
    a = np.ascontiguousarray(left.reshape(1067, w)[y0:y0 + h]).reshape(-1)
    b = np.ascontiguousarray(right.reshape(1067, w)[y0:y0 + h]).reshape(-1)
    o = Options()
    o.census, o.censusHeight, o.disparities = 9, 7, 128
    prm = params_from_options(o)
    prm.p1, prm.p2 = 10, 120
    want = orc.pair(prm, a, b, w, h, want_reasons=True)
    with GpuSgm(0) as s:
        resident = s.pair(prm, a, b, w, h, want_views=True, want_reasons=True)
        assert_same(resident, want, "resident")
        full = s.plan_detail(prm, w, h)
        assert not full["streamed"] and full["rows"] == h and full["host_bytes"] == 0
    with GpuSgm(0) as s:
        s.set_budget(full["device_bytes"] // 4)
        plan = s.plan_detail(prm, w, h)
        assert plan["streamed"] and (h + plan["rows"] - 1) // plan["rows"] >= 3
        assert plan["device_bytes"] <= full["device_bytes"] // 4
        got = s.pair(prm, a, b, w, h, want_views=True, want_reasons=True)
        assert_same(got, want, "streamed under a short budget")
        s.set_streaming("resident")
        with pytest.raises(_abi.CsgmError) as e:
            s.pair(prm, a, b, w, h)
        assert e.value.status == _abi.CSGM_E_NOMEM
        s.set_streaming("auto")
        again = s.pair(prm, a, b, w, h, want_views=True, want_reasons=True)
        assert_same(again, want, "streamed after a refused call")


@pytest.mark.parametrize("reverse", [0, 1])
def test_streamed_match_equals_oracle(session, reverse):
    """csgm_match (GpuSgm.match) streamed: one view with its winners records, reasons, flags."""
    from pose_b200.sgm import Stats

    w, h, a, b, ma, mb = scaling_pair()
    o = Options()
    o.disparities, o.minDisparity, o.directions = 33, -5, 16
    prm = params_from_options(o)
    da, db = orc.census(a, w, h, 5, 5), orc.census(b, w, h, 5, 5)
    ta = orc.texture(a, w, h, 5, 5) & (ma != 0)
    tb = orc.texture(b, w, h, 5, 5) & (mb != 0)
    if reverse:
        da, db, ta, tb, a, b = db, da, tb, ta, b, a
    n = w * h
    reasons_want, boundary_want = np.ones(n, np.uint8), np.zeros(n, np.uint8)
    want = orc.match(prm, da, db, a, b, ta, tb, w, h, reverse, want_summary=True,
                     reasons=reasons_want, boundary=boundary_want)
    session.set_streaming("streamed", 8)
    try:
        st = Stats()
        reasons, boundary = np.ones(n, np.uint8), np.zeros(n, np.uint8)
        disp, summary = session.match(prm, da, db, a, b, ta, tb, w, h, reverse, st, reasons,
                                      boundary, summary=True)
    finally:
        session.set_streaming("auto")
    assert np.array_equal(summary, want["summary"])
    assert np.array_equal(bits(disp), bits(want["disp"]))
    assert np.array_equal(reasons, reasons_want) and np.array_equal(boundary, boundary_want)
    s = want["stats"]
    assert (st.fullIntervalPixels, st.boundaryRejected, st.ambiguityRejected, st.selected) == (
        s.full_interval_pixels, s.boundary_rejected, s.ambiguity_rejected, s.selected)


def test_streaming_settings_are_checked(session):
    assert session.lib.csgm_session_set_streaming(session.handle, 4, 0) == _abi.CSGM_E_INVALID
    assert session.lib.csgm_session_set_streaming(session.handle, 0, -1) == _abi.CSGM_E_INVALID
    with pytest.raises(KeyError):
        session.set_streaming("disk")
