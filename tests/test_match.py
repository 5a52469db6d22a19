"""csgm_match, the drop-in for GpuSgm.match (GpuSgm.java:267-303), on the fused kernels.

CensusSgm.computeRecorded calls match(a, b, left, right, tl, tr, reverse=false, stats, reasons,
boundary) and then match(b, a, right, left, tr, tl, reverse=true, new Stats(), null, null)
(CensusSgm.java:135-162).  The library computes both views on the first call and answers the
mirrored second call from the view it kept, after checking on the device that the second call's
inputs are byte-identical.  Every result is compared with the oracle bit for bit.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle.oracle as orc
from pose_b200.options import Options
from pose_b200.stereo_cost import params_from_options

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def session():
    from pose_b200.sgm import GpuSgm

    orc.set_threads(8)
    s = GpuSgm(0)
    s.set_profiling(2)  # per-kernel records: which kernels each call launched
    yield s
    s.close()


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def views_inputs(left, right, w, h, wx, wy, ma=None, mb=None):
    da, db = orc.census(left, w, h, wx, wy), orc.census(right, w, h, wx, wy)
    ta = orc.texture(left, w, h, wx, wy)
    tb = orc.texture(right, w, h, wx, wy)
    if ma is not None:
        ta &= ma != 0
        tb &= mb != 0
    return da, db, ta, tb


def check_view(session, prm, inputs, w, h, reverse, want_summary=True):
    """One csgm_match call against the oracle's CensusSgm.match; returns the names of the kernels
    it launched."""
    from pose_b200.sgm import Stats

    da, db, ga, gb, ta, tb = inputs
    n = w * h
    reasons_want = np.ones(n, np.uint8) if not reverse else None
    boundary_want = np.zeros(n, np.uint8) if not reverse else None
    want = orc.match(prm, da, db, ga, gb, ta, tb, w, h, reverse, want_summary=True,
                     reasons=reasons_want, boundary=boundary_want)
    session.kernel_times(reset=True)
    st = Stats()
    reasons = np.ones(n, np.uint8) if not reverse else None
    boundary = np.zeros(n, np.uint8) if not reverse else None
    got = session.match(prm, da, db, ga, gb, ta, tb, w, h, reverse, st, reasons, boundary,
                        summary=want_summary)
    disp, summary = got if want_summary else (got, None)
    assert np.array_equal(bits(disp), bits(want["disp"])), f"reverse={reverse}: disparities"
    if want_summary:
        assert np.array_equal(summary, want["summary"]), f"reverse={reverse}: winners records"
    if not reverse:
        assert np.array_equal(reasons, reasons_want), "reason codes"
        assert np.array_equal(boundary, boundary_want), "boundary flags"
    s = want["stats"]
    assert (st.fullIntervalPixels, st.boundaryRejected, st.lowerBoundaryRejected,
            st.upperBoundaryRejected, st.ambiguityRejected, st.selected) == (
        s.full_interval_pixels, s.boundary_rejected, s.lower_boundary_rejected,
        s.upper_boundary_rejected, s.ambiguity_rejected, s.selected)
    return set(session.kernel_times(reset=True))


def band_inputs(wx=9, wy=7, rows=48):
    from pose_b200.synthetic import make_pair, spec_for

    left, right, _ = make_pair(spec_for("cfg1"))
    w, y0 = 1600, 500
    a = np.ascontiguousarray(left.reshape(1067, w)[y0:y0 + rows]).reshape(-1)
    b = np.ascontiguousarray(right.reshape(1067, w)[y0:y0 + rows]).reshape(-1)
    return a, b, w, rows


def band_params(wx=9, wy=7, D=128, directions=8, cost="census"):
    o = Options()
    o.census, o.censusHeight, o.disparities, o.directions = wx, wy, D, directions
    o.matchingCost = cost
    prm = params_from_options(o)
    prm.p1, prm.p2 = 10, 120
    return prm


@pytest.mark.parametrize("directions", [4, 8])
@pytest.mark.parametrize("cost", ["census", "census-gradient"])
def test_mirrored_call_is_answered_from_the_held_view(session, directions, cost):
    a, b, w, h = band_inputs()
    prm = band_params(directions=directions, cost=cost)
    da, db, ta, tb = views_inputs(a, b, w, h, 9, 7)
    first = check_view(session, prm, (da, db, a, b, ta, tb), w, h, 0)
    # The mirrored call (CensusSgm.java:149-162): inputs swapped, reverse=true.
    second = check_view(session, prm, (db, da, b, a, tb, ta), w, h, 1)
    assert {"cost_pair", "penalty", "sweep", "wta"} <= first
    assert second == {"bytes_differ"}, "the mirrored call should only compare its inputs"


def test_changed_input_is_recomputed(session):
    a, b, w, h = band_inputs()
    prm = band_params()
    da, db, ta, tb = views_inputs(a, b, w, h, 9, 7)
    check_view(session, prm, (da, db, a, b, ta, tb), w, h, 0)
    b2 = b.copy()
    b2[h // 2 * w + w // 2] ^= 0x5a  # one gray value of the target image differs
    second = check_view(session, prm, (db, da, b2, a, tb, ta), w, h, 1)
    assert "sweep" in second, "inputs differ from the held pair's: the view must be computed"


def test_reverse_first_and_general_in_between(session):
    """The held view follows the latest fused call; the general path keeps no view."""
    a, b, w, h = band_inputs(rows=40)
    prm = band_params(D=64)
    da, db, ta, tb = views_inputs(a, b, w, h, 9, 7)
    check_view(session, prm, (db, da, b, a, tb, ta), w, h, 1)   # right view first
    assert check_view(session, prm, (da, db, a, b, ta, tb), w, h, 0) == {"bytes_differ"}
    # no held view now: computed
    assert "sweep" in check_view(session, prm, (da, db, a, b, ta, tb), w, h, 0)
    prm.flags = 1  # CSGM_FLAG_GENERAL
    assert "paths_line" in check_view(session, prm, (db, da, b, a, tb, ta), w, h, 1)
    prm.flags = 0
    assert "sweep" in check_view(session, prm, (db, da, b, a, tb, ta), w, h, 1)


def test_masked_fixture_both_orders(session):
    """UpgradeStereoRegression's masked fixture (D=41, minD=-3), left then right view."""
    from fixtures import upgrade_pair

    w, h, _, a, b, ma, mb = upgrade_pair()
    o = Options()
    o.disparities, o.minDisparity = 41, -3
    prm = params_from_options(o)
    da, db, ta, tb = views_inputs(a, b, w, h, o.census, o.census, ma, mb)
    check_view(session, prm, (da, db, a, b, ta, tb), w, h, 0, want_summary=False)
    assert check_view(session, prm, (db, da, b, a, tb, ta), w, h, 1,
                      want_summary=False) == {"bytes_differ"}
