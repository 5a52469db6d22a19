"""Batched pairs (csgm_batch_*): every pair in a mix of uneven sizes, disparity ranges and cost
modes, run concurrently on several slots, is bit-identical to the same pair run alone through
csgm_pair; admission refuses a pair while the memory budget is held by pairs in flight and admits
it once they are collected."""
from __future__ import annotations

import numpy as np
import pytest

from pose_b200 import _abi
from pose_b200.batch import PairBatch
from pose_b200.options import Options
from pose_b200.stereo_cost import params_from_options
from pose_b200.synthetic import PairSpec, make_pair

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def mixed_pairs():
    """Six pairs: widths 200..420, aspect 3:2 / 4:3, D in {64, 128, 192, 256}, census and
    AD-census, 8 and 4 paths."""
    cases = [(320, 214, 64, "census", 8), (420, 280, 128, "ad-census", 8),
             (240, 180, 192, "census", 4), (360, 270, 256, "census", 8),
             (200, 150, 128, "census-gradient", 8), (300, 200, 64, "ad-census", 4)]
    out = []
    for i, (w, h, d, cost, dirs) in enumerate(cases):
        spec = PairSpec(w, h, planes=3, d_min=2, d_max=max(4, d // 2), seed=100 + i)
        left, right, _ = make_pair(spec)
        o = Options()
        o.census, o.censusHeight, o.disparities = 9, 7, d
        o.matchingCost, o.directions = cost, dirs
        prm = params_from_options(o)
        prm.p1, prm.p2 = 10, 120
        out.append((prm, left, right, w, h))
    return out


@pytest.fixture(scope="module")
def session():
    from pose_b200.sgm import GpuSgm

    s = GpuSgm(0)
    yield s
    s.close()


def test_batched_equals_alone(session):
    pairs = mixed_pairs()
    alone = [session.pair(prm, l, r, w, h, want_views=True, want_reasons=True)
             for prm, l, r, w, h in pairs]
    batch = PairBatch(session, slots=3)
    pending, results = list(range(len(pairs))), {}
    ids = {}
    while pending or ids:
        while pending:  # submit while admission allows
            i = pending[0]
            prm, l, r, w, h = pairs[i]
            rid = batch.submit(prm, l, r, w, h, want_views=True, want_reasons=True)
            if rid is None:
                break
            ids[rid] = i
            pending.pop(0)
        rid = next(iter(ids))
        results[ids.pop(rid)] = batch.poll(rid, wait=True)
    for i, want in enumerate(alone):
        got = results[i]
        assert np.array_equal(bits(got.disparity), bits(want.disparity)), f"pair {i}: LR-checked"
        assert np.array_equal(bits(got.left), bits(want.left)), f"pair {i}: left view"
        assert np.array_equal(bits(got.right), bits(want.right)), f"pair {i}: right view"
        assert np.array_equal(got.reasons, want.reasons), f"pair {i}: reasons"
        assert np.array_equal(got.searchBoundary, want.searchBoundary), f"pair {i}: boundary"
        assert got.stats == want.stats, f"pair {i}: counters"
    assert batch.status()["in_flight"] == 0


def test_admission_waits_for_memory(session):
    prm, l, r, w, h = mixed_pairs()[1]
    need = session.plan(prm, w, h)
    batch = PairBatch(session, slots=4, budget_bytes=int(need * 1.5))
    first = batch.submit(prm, l, r, w, h)
    assert first is not None
    assert batch.submit(prm, l, r, w, h) is None  # the budget is held by the first pair
    assert batch.status()["reserved_bytes"] == need
    first_result = batch.poll(first, wait=True)
    second = batch.submit(prm, l, r, w, h)  # admitted once the first is collected
    assert second is not None
    second_result = batch.poll(second, wait=True)
    assert np.array_equal(bits(first_result.disparity), bits(second_result.disparity))


def test_poll_unknown_request(session):
    batch = PairBatch(session, slots=1)
    with pytest.raises(_abi.CsgmError) as err:
        batch.poll(123456789)
    assert err.value.status == _abi.CSGM_E_INVALID
