"""Compact SGM (--gpu-sgm esgm, GpuCandidateStereo.java:53-167): per-path proposals, compact
aggregates with a lower bound elsewhere, certification, and the exact pass over the pixels the
proposals do not certify.  The outcome is the full SGM's: every result is compared with the oracle
bit for bit, including the exact pass in chunks under a short budget.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle.oracle as orc
from fixtures import esgm_production_pair, scaling_pair, upgrade_pair
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


def compact_pair(s, prm, a, b, w, h, ma=None, mb=None, pool=2):
    s.set_streaming("esgm")
    s.set_candidates(pool)
    try:
        plan = s.plan_detail(prm, w, h)
        assert not plan["streamed"] and plan["host_bytes"] == 0
        got = s.pair(prm, a, b, w, h, ma, mb, want_views=True, want_reasons=True)
        reports = [s.compact_report(r) for r in (0, 1)]
    finally:
        s.set_streaming("auto")
        s.set_candidates(2)
    for certified, verified in reports:
        assert certified + verified == w * h and verified >= 0
    return got, reports


@pytest.mark.parametrize("pool", [1, 2, 4])
@pytest.mark.parametrize("directions", [4, 8, 16])
def test_compact_pair_equals_oracle(session, pool, directions):
    """UpgradeStereoRegression's masked fixture (192x79, D41, minD -3)."""
    w, h, _, a, b, ma, mb = upgrade_pair()
    o = Options()
    o.disparities, o.minDisparity, o.directions = 41, -3, directions
    prm = params_from_options(o)
    want = orc.pair(prm, a, b, w, h, ma, mb, want_reasons=True)
    got, _ = compact_pair(session, prm, a, b, w, h, ma, mb, pool)
    assert_same(got, want, f"compact {directions}-path, {pool} proposals per path")


@pytest.mark.parametrize("fixture", [0, 1, 2])
@pytest.mark.parametrize("directions", [4, 8])
def test_production_fixtures(session, fixture, directions):
    """EsgmProductionRegression (EsgmProductionRegression.java:15-65): D129 from -15, noise, a
    periodic pattern and a negative shift; compact with 1, 2 and 4 proposals per path equals the
    resident views (and the oracle) in every output and counter."""
    w, h, a, b, ma, mb = esgm_production_pair(fixture)
    o = Options()
    o.minDisparity, o.disparities, o.directions = -15, 129, directions
    o.median, o.speckleSize = 1, 0
    prm = params_from_options(o)
    want = orc.pair(prm, a, b, w, h, ma, mb, want_reasons=True)
    session.set_streaming("resident")
    try:
        resident = session.pair(prm, a, b, w, h, ma, mb, want_views=True, want_reasons=True)
    finally:
        session.set_streaming("auto")
    assert_same(resident, want, "resident")
    for pool in (1, 2, 4):
        got, _ = compact_pair(session, prm, a, b, w, h, ma, mb, pool)
        assert_same(got, want, f"fixture {fixture}, {directions} paths, {pool} proposals")


def test_wide_disparity_range(session):
    """D = 2100 (the path kernels then run two warps a block to fit four D-rows each in shared
    memory) on a 2304x9 noise pair shifted by 1500."""
    from fixtures import shifted

    w, h = 2304, 9
    a = np.random.default_rng(31).integers(0, 256, w * h, dtype=np.uint8)
    b = shifted(a, w, h, 1500)
    o = Options()
    o.disparities, o.directions, o.census = 2100, 4, 3
    prm = params_from_options(o)
    want = orc.pair(prm, a, b, w, h, want_reasons=True)
    got, _ = compact_pair(session, prm, a, b, w, h, pool=1)
    assert_same(got, want, "compact, D2100")


def test_compact_crop_equals_oracle(session):
    """A 1600x200 crop of the synthetic 1600x1067 scene (D128, census 9x7): one proposal per path
    leaves pixels to the exact pass, which must then give the full SGM's outcome."""
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
    for pool in (1, 2):
        got, reports = compact_pair(session, prm, a, b, w, h, pool=pool)
        assert_same(got, want, f"compact crop, {pool} proposals per path")
        if pool == 1:
            assert all(verified > 0 for _, verified in reports)


def test_exact_pass_in_chunks():
    """A budget of exactly the compact plan leaves one image row of exact aggregates: the exact
    pass runs in many chunks and still equals the oracle; a budget below the smallest plan is
    refused."""
    from pose_b200.sgm import GpuSgm

    # Two unrelated noise images: few outcomes are certain, so most pixels go to the exact pass.
    w, h = 160, 47
    rng = np.random.default_rng(20)
    a = rng.integers(0, 256, w * h, dtype=np.uint8)
    b = rng.integers(0, 256, w * h, dtype=np.uint8)
    o = Options()
    o.disparities, o.minDisparity, o.directions = 33, -5, 8
    prm = params_from_options(o)
    want = orc.pair(prm, a, b, w, h, want_reasons=True)
    with GpuSgm(0) as s:
        s.set_streaming("esgm")
        s.set_candidates(1)
        plan = s.plan_detail(prm, w, h)
    with GpuSgm(0) as s:
        s.set_budget(plan["device_bytes"])
        got, reports = compact_pair(s, prm, a, b, w, h, pool=1)
        assert_same(got, want, "compact with one row of exact aggregates")
        assert max(v for _, v in reports) > w, "the exact pass should take several chunks"
    # The smallest plan holds one view's arrays at a time (8 bytes per path and pixel + 12).
    smallest = plan["device_bytes"] - w * h * (prm.directions * 8 + 12)
    with GpuSgm(0) as s:
        s.set_streaming("esgm")
        s.set_candidates(1)
        s.set_budget(smallest)
        assert s.plan_detail(prm, w, h)["device_bytes"] == smallest
        s.set_budget(smallest - 1)
        with pytest.raises(_abi.CsgmError) as e:
            s.pair(prm, a, b, w, h)
        assert e.value.status == _abi.CSGM_E_NOMEM


def test_plan_lowers_the_proposals_to_fit():
    """GpuCandidateStereo.plan tries pool = esgmCandidates .. 1: a budget between the 1- and
    2-proposal plans gives the 1-proposal plan.  A pair's plan first holds both views' arrays;
    below the smallest such plan it runs one view after the other."""
    from pose_b200.sgm import GpuSgm

    w, h, _, a, b, ma, mb = upgrade_pair()
    n = w * h
    o = Options()
    o.disparities, o.minDisparity = 41, -3
    prm = params_from_options(o)
    want = orc.pair(prm, a, b, w, h, ma, mb, want_reasons=True)
    per_view = {pool: n * (prm.directions * pool * 8 + 12) for pool in (1, 2)}
    with GpuSgm(0) as s:
        s.set_streaming("esgm")
        sizes = {}
        for pool in (1, 2):
            s.set_candidates(pool)
            sizes[pool] = s.plan_detail(prm, w, h)["device_bytes"]
        assert sizes[2] - sizes[1] == 2 * (per_view[2] - per_view[1])  # both views' arrays
        s.set_budget(sizes[2] - 1)
        s.set_candidates(2)
        assert s.plan_detail(prm, w, h)["device_bytes"] == sizes[1]
        got = s.pair(prm, a, b, w, h, ma, mb, want_views=True, want_reasons=True)
        assert_same(got, want, "compact with the lowered proposal count")
        one_view = sizes[2] - per_view[2]  # 2 proposals, one view's arrays
        assert one_view < sizes[1]
        s.set_budget(sizes[1] - 1)
        assert s.plan_detail(prm, w, h)["device_bytes"] == one_view
        got = s.pair(prm, a, b, w, h, ma, mb, want_views=True, want_reasons=True)
        assert_same(got, want, "compact one view after the other")
        assert all(c + v == n for c, v in (s.compact_report(r) for r in (0, 1)))


@pytest.mark.parametrize("reverse", [0, 1])
def test_compact_match_equals_oracle(session, reverse):
    """csgm_match (GpuSgm.match) in compact mode: disparities, reasons, flags and counters equal the
    oracle; the winners records equal it except a certified pixel's second value, which is the best
    known one and so never below the exact one."""
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
    session.set_streaming("esgm")
    try:
        st = Stats()
        reasons, boundary = np.ones(n, np.uint8), np.zeros(n, np.uint8)
        disp, summary = session.match(prm, da, db, a, b, ta, tb, w, h, reverse, st, reasons,
                                      boundary, summary=True)
    finally:
        session.set_streaming("auto")
    assert np.array_equal(bits(disp), bits(want["disp"]))
    assert np.array_equal(reasons, reasons_want) and np.array_equal(boundary, boundary_want)
    s = want["stats"]
    assert (st.fullIntervalPixels, st.boundaryRejected, st.ambiguityRejected, st.selected) == (
        s.full_interval_pixels, s.boundary_rejected, s.ambiguity_rejected, s.selected)
    got, ref = summary.reshape(n, 6), want["summary"].reshape(n, 6)
    exact = [0, 1, 3, 4, 5]
    assert np.array_equal(got[:, exact], ref[:, exact])
    assert np.all(got[:, 2] >= ref[:, 2])


def test_compact_settings_are_checked(session):
    lib, hd = session.lib, session.handle
    assert lib.csgm_session_set_candidates(hd, 0) == _abi.CSGM_E_INVALID
    assert lib.csgm_session_set_candidates(hd, 5) == _abi.CSGM_E_INVALID
    assert lib.csgm_session_set_streaming(hd, 4, 0) == _abi.CSGM_E_INVALID
    assert lib.csgm_session_compact_report(hd, 2, None, None) == _abi.CSGM_E_INVALID
    w, h, _, a, b, ma, mb = upgrade_pair()
    session.set_streaming("esgm")
    try:
        for cost, agg in (("zncc", "16"), ("census", "32")):
            o = Options()
            o.disparities, o.matchingCost, o.sgmAggregate = 41, cost, agg
            prm = params_from_options(o)
            with pytest.raises(_abi.CsgmError) as e:
                session.pair(prm, a, b, w, h, ma, mb)
            assert e.value.status == _abi.CSGM_E_INVALID
    finally:
        session.set_streaming("auto")


def test_census_sgm_compute_in_compact_mode(session):
    """CensusSgm.compute with Options.gpuSgm = "esgm" (the matcher, the LR check and every
    post-filter on its outputs) equals the resident run: the map, reasons and the Stats CSV."""
    from pose_b200.sgm import CensusSgm

    w, h, a, b, ma, mb = esgm_production_pair(0)
    results = {}
    for mode, pool in (("resident", 2), ("esgm", 1), ("esgm", 4)):
        o = Options()
        o.minDisparity, o.disparities, o.directions = -15, 129, 8
        o.gpuSgm, o.esgmCandidates = mode, pool
        results[(mode, pool)] = CensusSgm(o, session=session).compute(a, b, w, h, ma, mb,
                                                                     want_reasons=True)
    session.set_streaming("auto")
    session.set_candidates(2)
    want = results[("resident", 2)]
    for key in (("esgm", 1), ("esgm", 4)):
        got = results[key]
        assert np.array_equal(bits(got.disparity), bits(want.disparity)), key
        assert np.array_equal(got.reasons, want.reasons), key
        assert got.stats.csv() == want.stats.csv(), key


def test_auto_runs_compact_over_the_host_budget():
    """GpuStereo.execute (GpuStereo.java:184-193) under --gpu-sgm auto: a pair over the device
    budget streams while its aggregate fits the host budget, and runs compact SGM (no host bytes,
    the same results) once it does not; streamed mode refuses instead."""
    from pose_b200.sgm import GpuSgm

    w, h, _, a, b, ma, mb = upgrade_pair()
    o = Options()
    o.disparities, o.minDisparity = 41, -3
    prm = params_from_options(o)
    want = orc.pair(prm, a, b, w, h, ma, mb, want_reasons=True)
    with GpuSgm(0) as s:
        full = s.plan_detail(prm, w, h)
        s.set_budget(full["device_bytes"] // 3)
        streamed = s.plan_detail(prm, w, h)
        assert streamed["streamed"] and streamed["host_bytes"] > 0
        s.set_host_budget(streamed["host_bytes"])
        assert s.plan_detail(prm, w, h) == streamed
        s.set_host_budget(streamed["host_bytes"] - 1)
        compact = s.plan_detail(prm, w, h)
        assert not compact["streamed"] and compact["host_bytes"] == 0
        got = s.pair(prm, a, b, w, h, ma, mb, want_views=True, want_reasons=True)
        assert_same(got, want, "auto over the host budget")
        assert all(c + v == w * h and c > 0 for c, v in (s.compact_report(r) for r in (0, 1)))
        s.set_streaming("streamed", 16)
        with pytest.raises(_abi.CsgmError) as e:
            s.pair(prm, a, b, w, h, ma, mb)
        assert e.value.status == _abi.CSGM_E_NOMEM
        s.set_streaming("auto")
        zncc = params_from_options(Options(disparities=41, minDisparity=-3, matchingCost="zncc"))
        with pytest.raises(_abi.CsgmError) as e:  # compact SGM is Census only
            s.pair(zncc, a, b, w, h, ma, mb)
        assert e.value.status == _abi.CSGM_E_NOMEM
        s.set_host_budget(0)
        again = s.pair(prm, a, b, w, h, ma, mb, want_views=True, want_reasons=True)
        assert_same(again, want, "streamed again without a host budget")


def test_plan_switch_frees_the_other_plans_buffers():
    """A session's workspace keeps its buffers from call to call. A compact call after a resident
    one frees the resident volumes, so it fits a budget of exactly its own plan; the resident call
    after it frees the compact arrays again."""
    from pose_b200.sgm import GpuSgm

    w, h, _, a, b, ma, mb = upgrade_pair()
    o = Options()
    o.disparities, o.minDisparity = 41, -3
    prm = params_from_options(o)
    want = orc.pair(prm, a, b, w, h, ma, mb, want_reasons=True)
    with GpuSgm(0) as s:
        assert_same(s.pair(prm, a, b, w, h, ma, mb, want_views=True, want_reasons=True), want,
                    "resident")
        resident_bytes = s.plan_detail(prm, w, h)["device_bytes"]
        s.set_streaming("esgm")
        s.set_budget(s.plan_detail(prm, w, h)["device_bytes"])
        assert_same(s.pair(prm, a, b, w, h, ma, mb, want_views=True, want_reasons=True), want,
                    "compact after resident")
        s.set_streaming("auto")
        s.set_budget(resident_bytes)
        assert_same(s.pair(prm, a, b, w, h, ma, mb, want_views=True, want_reasons=True), want,
                    "resident after compact")
