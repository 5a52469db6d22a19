"""CUDA matcher == CPU oracle, bit for bit, on the reference's own CPU==GPU fixtures.

Restates StorageGpuRegression.java:68-104, ScalingRegression.java:56-99 and
UpgradeStereoRegression.java:35-80,98-125 with "GPU" = libcollinea_sgm.so through the C ABI and
"CPU" = the oracle.  Disparities are compared as raw float bits (subpixel values are bit-exact,
far inside the 1e-4 px tolerance), counters and per-pixel reason codes exactly.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle.oracle as orc
from fixtures import (scaling_pair, storage_gpu_pair, upgrade_large_pair, upgrade_pair)
from pose_b200 import _abi
from pose_b200.options import Options
from pose_b200.stereo_cost import params_from_options

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def session():
    from pose_b200.sgm import GpuSgm

    orc.set_threads(8)
    s = GpuSgm(0)
    yield s
    s.close()


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def stats_tuple(s):
    return tuple(int(getattr(s, k)) for k in _abi.STATS_FIELDS)


GENERAL = 1  # CSGM_FLAG_GENERAL


def assert_pair_equal(session, o, a, b, w, h, ma=None, mb=None, params=None):
    """Both GPU paths (the fused sweep where it applies, and the general kernels) == oracle."""
    prm = params if params is not None else params_from_options(o)
    want = orc.pair(prm, a, b, w, h, ma, mb, want_reasons=True)
    got = None
    for flags in (0, GENERAL):
        prm.flags = flags
        got = session.pair(prm, a, b, w, h, ma, mb, want_views=True, want_reasons=True)
        path = "general" if flags else "default"
        assert np.array_equal(bits(got.left), bits(want["dl"])), f"{path}: left view disparities"
        assert np.array_equal(bits(got.right), bits(want["dr"])), f"{path}: right view"
        assert np.array_equal(bits(got.disparity), bits(want["checked"])), f"{path}: LR-checked"
        assert np.array_equal(got.reasons, want["reasons"]), f"{path}: reason codes"
        assert np.array_equal(got.searchBoundary, want["boundary"]), f"{path}: boundary flags"
        assert stats_tuple(got.stats.to_c()) == stats_tuple(want["stats"]), f"{path}: counters"
    prm.flags = 0
    return got


@pytest.mark.parametrize("cost", ["census", "ad-census", "census-gradient", "zncc"])
@pytest.mark.parametrize("directions,agg", [(4, "16"), (8, "16"), (4, "32"), (8, "32")])
@pytest.mark.parametrize("reverse", [0, 1])
def test_match_scaling_fixture(session, cost, directions, agg, reverse):
    """csgm_match (GpuSgm.match drop-in) on ScalingRegression's fixture: D=33, minD=-5."""
    w, h, a, b, ma, mb = scaling_pair()
    o = Options()
    o.disparities, o.minDisparity = 33, -5
    o.matchingCost, o.directions, o.sgmAggregate = cost, directions, agg
    prm = params_from_options(o)
    da, db = orc.census(a, w, h, 5, 5), orc.census(b, w, h, 5, 5)
    ta = orc.texture(a, w, h, 5, 5) & (ma != 0)
    tb = orc.texture(b, w, h, 5, 5) & (mb != 0)
    if reverse:
        da, db, ta, tb, a, b = db, da, tb, ta, b, a
    n = w * h
    reasons_want = np.ones(n, np.uint8)
    boundary_want = np.zeros(n, np.uint8)
    want = orc.match(prm, da, db, a, b, ta, tb, w, h, reverse, want_summary=True,
                     reasons=reasons_want, boundary=boundary_want)
    from pose_b200.sgm import Stats

    for flags in (0, GENERAL):  # the fused kernels where they apply, and the general ones
        prm.flags = flags
        st = Stats()
        reasons = np.ones(n, np.uint8)
        boundary = np.zeros(n, np.uint8)
        disp, summary = session.match(prm, da, db, a, b, ta, tb, w, h, reverse, st, reasons,
                                      boundary, summary=True)
        assert np.array_equal(summary, want["summary"]), "winners record"
        assert np.array_equal(bits(disp), bits(want["disp"]))
        assert np.array_equal(reasons, reasons_want) and np.array_equal(boundary, boundary_want)
        s = want["stats"]
        assert (st.fullIntervalPixels, st.boundaryRejected, st.lowerBoundaryRejected,
                st.upperBoundaryRejected, st.ambiguityRejected, st.selected) == (
            s.full_interval_pixels, s.boundary_rejected, s.lower_boundary_rejected,
            s.upper_boundary_rejected, s.ambiguity_rejected, s.selected)
    prm.flags = 0


@pytest.mark.parametrize("census", [5, 11])
@pytest.mark.parametrize("directions", [4, 8])
def test_pair_storage_fixture(session, census, directions):
    """StorageGpuRegression.java:68-90 (gray mode): D=37 (5x5) or 177 (11x11), masked hole."""
    w, h, a, b, mask = storage_gpu_pair()
    o = Options()
    o.census, o.directions = census, directions
    o.disparities = 177 if census == 11 else 37
    assert_pair_equal(session, o, a, b, w, h, mask, mask)


def test_pair_signed_range(session):
    """StorageGpuRegression.java:91-104: D=29, minDisparity -16, swapped images."""
    w, h, a, b, _ = storage_gpu_pair()
    o = Options()
    o.disparities, o.minDisparity = 29, -16
    assert_pair_equal(session, o, b, a, w, h)


@pytest.mark.parametrize("cost", ["census", "ad-census", "census-gradient", "zncc"])
@pytest.mark.parametrize("directions", [4, 8])
def test_pair_upgrade_fixture(session, cost, directions):
    """UpgradeStereoRegression.java:35-80: D=41, minD=-3, masks on both sides."""
    w, h, shift, a, b, ma, mb = upgrade_pair()
    o = Options()
    o.disparities, o.minDisparity = 41, -3
    o.matchingCost, o.directions = cost, directions
    assert_pair_equal(session, o, a, b, w, h, ma, mb)


def test_pair_693_hypotheses(session):
    """UpgradeStereoRegression.java:98-125: 800x64, D=693 (many banks in the reference)."""
    w, h, a, b = upgrade_large_pair()
    o = Options()
    o.disparities = 693
    assert_pair_equal(session, o, a, b, w, h)


@pytest.mark.parametrize("wx,wy,cost", [(9, 7, "census"), (9, 7, "census-gradient"),
                                        (9, 9, "census"), (7, 7, "zncc"), (7, 7, "ad-census")])
def test_pair_synthetic_windows(session, wx, wy, cost):
    """The benchmark's window/cost combinations on a small synthetic pair (9x7 is the
    rectangular extension; its square special cases are the reference's)."""
    from pose_b200.synthetic import PairSpec, make_pair

    spec = PairSpec(224, 96, planes=3, d_min=4, d_max=40, seed=7)
    a, b, _ = make_pair(spec)
    o = Options()
    o.census, o.censusHeight, o.matchingCost, o.disparities = wx, wy, cost, 48
    prm = params_from_options(o)
    prm.p1, prm.p2 = 10, 120
    assert_pair_equal(session, o, a, b, spec.width, spec.height, params=prm)


def test_pair_uint32_large_penalty(session):
    """P2 large enough that path costs exceed 16 bits: the uint32 aggregate and int32 path state."""
    w, h, a, b, ma, mb = scaling_pair()
    o = Options()
    o.disparities, o.p1, o.p2 = 20, 100, 40000
    o.sgmEdgeScale = 0
    prm = params_from_options(o)
    assert prm.aggregate_bytes == 4 and prm.p2 > 32000
    assert_pair_equal(session, o, a, b, w, h, ma, mb, params=prm)


def test_invalid_arguments_are_rejected(session):
    prm = params_from_options(Options())
    img = np.zeros(64 * 48, np.uint8)
    bad = params_from_options(Options())
    bad.directions = 6
    with pytest.raises(_abi.CsgmError) as e:
        session.pair(bad, img, img, 64, 48)
    assert e.value.status == _abi.CSGM_E_INVALID
    tiny = np.zeros(6 * 6, np.uint8)
    with pytest.raises(_abi.CsgmError) as e:  # smaller than census + 2 (CensusSgm.java:56-60)
        session.pair(prm, tiny, tiny, 6, 6)
    assert e.value.status == _abi.CSGM_E_INVALID
    with pytest.raises(ValueError):  # buffer size does not match w*h
        session.pair(prm, img, img, 6, 6)


def test_budget_rejects_before_allocation():
    """StorageGpuRegression.java:135-144: an impossible budget is refused before any work."""
    from pose_b200.sgm import GpuSgm

    with GpuSgm(0, memory_mb=1) as s:
        s.set_streaming("resident")  # the reference test's --gpu-sgm resident
        w, h, a, b, _ = storage_gpu_pair()
        prm = params_from_options(Options())
        with pytest.raises(_abi.CsgmError) as e:
            s.pair(prm, a, b, w, h)
        assert e.value.status == _abi.CSGM_E_NOMEM
        limit = s.disparityLimit(prm, w, h)  # GpuStereo.limit: largest D whose plan fits
        assert 0 <= limit < prm.disparities
        if limit >= 3:
            prm.disparities = limit
            s.plan(prm, w, h)
            prm.disparities = limit + 1
            with pytest.raises(_abi.CsgmError):
                s.plan(prm, w, h)
        prm = params_from_options(Options())
    with GpuSgm(0) as s:
        assert s.disparityLimit(prm, w, h) == 4096
        # the session stays usable after a rejected call
        s.pair(prm, a, b, w, h)


def test_repeatable(session):
    w, h, a, b, mask = storage_gpu_pair()
    prm = params_from_options(Options())
    r1 = session.pair(prm, a, b, w, h, mask, mask)
    r2 = session.pair(prm, a, b, w, h, mask, mask)
    assert np.array_equal(bits(r1.disparity), bits(r2.disparity))


def bench_params(wx=9, wy=7, D=128, cost="census"):
    o = Options()
    o.census, o.censusHeight, o.disparities, o.matchingCost = wx, wy, D, cost
    prm = params_from_options(o)
    prm.p1, prm.p2 = 10, 120
    return prm


@pytest.mark.parametrize("D", [64, 128, 192, 256])
def test_pair_band_of_cfg1(session, D):
    """A full-width 1600 x 48 band of the benchmark pair, every fused register layout, vs oracle."""
    from pose_b200.synthetic import make_pair, spec_for

    left, right, _ = make_pair(spec_for("cfg1"))
    w, h = 1600, 48
    y0 = 500
    band_l = np.ascontiguousarray(left.reshape(1067, w)[y0:y0 + h]).reshape(-1)
    band_r = np.ascontiguousarray(right.reshape(1067, w)[y0:y0 + h]).reshape(-1)
    o = Options()
    o.census, o.censusHeight = 9, 7
    assert_pair_equal(session, o, band_l, band_r, w, h, params=bench_params(D=D))


@pytest.fixture(scope="module")
def oracle_threads():
    """The full-size oracle runs use every host core (a cfg1 pair takes a few seconds)."""
    import os

    orc.set_threads(os.cpu_count() or 8)
    yield
    orc.set_threads(8)


@pytest.mark.parametrize("cost", ["census", "census-gradient"])
def test_full_size_cfg1_equals_oracle(session, oracle_threads, cost):
    """The 1600x1067 D128 Census 9x7 benchmark pair, whole, on both GPU paths against the oracle:
    left and right views, LR-checked map, reasons, boundary flags and counters bit for bit.  The
    LR-checked map also recovers the synthetic ground truth."""
    from pose_b200.synthetic import make_pair, spec_for

    spec = spec_for("cfg1")
    left, right, truth = make_pair(spec)
    o = Options()
    o.census, o.censusHeight = 9, 7
    got = assert_pair_equal(session, o, left, right, spec.width, spec.height,
                            params=bench_params(cost=cost))
    d = got.disparity
    ok = np.isfinite(d)
    assert ok.mean() > 0.5
    assert (np.abs(d[ok] - truth[ok]) < 1.0).mean() > 0.9


@pytest.mark.parametrize("wx,wy,edge_scale", [(9, 9, 32), (9, 7, 32), (9, 9, 0)])
def test_full_size_cfg0_equals_oracle(session, oracle_threads, wx, wy, edge_scale):
    """The 640x480 D64 CPU-runnable workload, whole: Census 9x9 with Options p1=3 / p2=36 (the
    effective P1=10 / P2=120 of 80-bit descriptors, StereoCost.java:17-23), the 9x7 extension
    with the effective penalties given directly, and constant P2 (sgmEdgeScale 0)."""
    from pose_b200.synthetic import make_pair, spec_for

    spec = spec_for("cfg0")
    left, right, truth = make_pair(spec)
    o = Options()
    o.census, o.censusHeight, o.disparities = wx, wy, 64
    o.sgmEdgeScale = edge_scale
    if wx == wy:
        o.p1, o.p2 = 3, 36
        prm = params_from_options(o)
        assert (prm.p1, prm.p2) == (10, 120)
    else:
        prm = params_from_options(o)
        prm.p1, prm.p2 = 10, 120
    got = assert_pair_equal(session, o, left, right, spec.width, spec.height, params=prm)
    d = got.disparity
    ok = np.isfinite(d)
    assert ok.mean() > 0.5
    assert (np.abs(d[ok] - truth[ok]) < 1.0).mean() > 0.85


def test_full_size_repeatable(session):
    from pose_b200.synthetic import make_pair, spec_for

    spec = spec_for("cfg1")
    left, right, _ = make_pair(spec)
    prm = bench_params()
    r1 = session.pair(prm, left, right, spec.width, spec.height)
    r2 = session.pair(prm, left, right, spec.width, spec.height)
    assert np.array_equal(bits(r1.disparity), bits(r2.disparity))
    assert r1.stats == r2.stats


@pytest.mark.parametrize("cost", ["census", "ad-census", "zncc"])
@pytest.mark.parametrize("agg", ["16", "32"])
def test_pair_16_paths_fixture(session, cost, agg):
    """The 16-path extension (the eight (+-1,+-2), (+-2,+-1) directions after the reference's
    eight) on UpgradeStereoRegression's masked fixture, uint16 and uint32 aggregates."""
    w, h, shift, a, b, ma, mb = upgrade_pair()
    o = Options()
    o.disparities, o.minDisparity = 41, -3
    o.matchingCost, o.directions, o.sgmAggregate = cost, 16, agg
    prm = params_from_options(o)
    assert prm.aggregate_bytes == (2 if agg == "16" else 4)
    assert_pair_equal(session, o, a, b, w, h, ma, mb, params=prm)


def cfg2_params(cost):
    """The 3000x2000 workload: window 7x7, D256, 16 paths, uint32 forced; AD-Census lambda_AD 10
    as --ad-truncation 10 with census weight 0.5; ZNCC 7x7 (cost scale 0..48); the reference's
    default penalties (p1 4, p2 24 in 5x5 units: effective 8 / 48 at 48 bits)."""
    o = Options()
    o.census = 7
    o.disparities, o.directions, o.sgmAggregate = 256, 16, "32"
    o.matchingCost, o.adTruncation, o.censusWeight = cost, 10, 0.5
    prm = params_from_options(o)
    assert prm.aggregate_bytes == 4 and (prm.p1, prm.p2) == (8, 48)
    return o, prm


@pytest.mark.parametrize("cost", ["ad-census", "zncc"])
def test_pair_band_of_cfg2(session, oracle_threads, cost):
    """A full-width 3000 x 32 band of the 3000x2000 pair (10 planes, saturated specular patches)
    against the oracle: 16 paths, uint32 aggregate, D256."""
    from pose_b200.synthetic import make_pair, spec_for

    spec = spec_for("cfg2")
    left, right, _ = make_pair(spec)
    w, h, y0 = spec.width, 32, 900
    band_l = np.ascontiguousarray(left.reshape(spec.height, w)[y0:y0 + h]).reshape(-1)
    band_r = np.ascontiguousarray(right.reshape(spec.height, w)[y0:y0 + h]).reshape(-1)
    o, prm = cfg2_params(cost)
    assert_pair_equal(session, o, band_l, band_r, w, h, params=prm)
