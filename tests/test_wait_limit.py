"""The sweep's bounded device-side waits: a wait that runs out ends the call with CSGM_E_TIMEOUT
and a site code, no copy is left in flight, and the next call on the same session is bit-exact.

No fault is injected: a watchdog of one SM clock cycle makes the first wait that is not already
satisfied give up (the publisher warp of every row block but the last waits for its own rows'
first carry chunk, which takes at least a dozen pixel steps).  The reference has no device-side
wait to bound (its host blocks in clFinish, GpuSgm.java:606-609).
"""
from __future__ import annotations

import re

import numpy as np
import pytest

import oracle.oracle as orc
from pose_b200 import _abi
from pose_b200.options import Options
from pose_b200.stereo_cost import params_from_options

pytestmark = pytest.mark.gpu


def small_pair():
    from pose_b200.synthetic import PairSpec, make_pair

    spec = PairSpec(320, 160, planes=3, d_min=4, d_max=40, seed=23)
    left, right, _ = make_pair(spec)
    return spec.width, spec.height, left, right


@pytest.mark.parametrize("directions", [4, 8])
def test_expired_wait_returns_timeout_and_session_recovers(directions):
    from pose_b200.sgm import GpuSgm

    w, h, left, right = small_pair()
    o = Options()
    o.census, o.censusHeight, o.disparities, o.directions = 9, 7, 64, directions
    prm = params_from_options(o)
    prm.p1, prm.p2 = 10, 120
    want = orc.pair(prm, left, right, w, h, want_reasons=True)
    with GpuSgm(0) as s:
        for attempt in range(2):  # twice in a row: the error word is reset between calls
            s.set_wait_limit(1)
            with pytest.raises(_abi.CsgmError) as e:
                s.pair(prm, left, right, w, h)
            assert e.value.status == _abi.CSGM_E_TIMEOUT
            code = int(re.search(r"code (\d+)", str(e.value)).group(1))
            assert code in (1, 3, 5, 6), str(e.value)
            s.set_wait_limit(0)
            got = s.pair(prm, left, right, w, h, want_views=True, want_reasons=True)
            assert np.array_equal(got.disparity.view(np.uint32), want["checked"].view(np.uint32))
            assert np.array_equal(got.left.view(np.uint32), want["dl"].view(np.uint32))
            assert np.array_equal(got.right.view(np.uint32), want["dr"].view(np.uint32))
            assert np.array_equal(got.reasons, want["reasons"])


def test_wait_limit_rejects_negative():
    from pose_b200.sgm import GpuSgm

    with GpuSgm(0) as s:
        with pytest.raises(_abi.CsgmError) as e:
            s.set_wait_limit(-1)
        assert e.value.status == _abi.CSGM_E_INVALID
