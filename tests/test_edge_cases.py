"""Edge cases against the oracle, bit for bit on both kernel paths and, where it applies
(Census, 16-bit aggregates), through compact SGM: the smallest image the reference accepts
(CensusSgm.java:56-60), the smallest and largest disparity counts, ranges at the fused kernels'
edge, odd sizes, everything masked out, large negative ranges, and an image taller than the fused
sweep's row limit (65535 rows: the general kernels run it)."""
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
    yield s
    s.close()


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def check(session, o, a, b, w, h, ma=None, mb=None, paths=(0, 1)):
    prm = params_from_options(o)
    want = orc.pair(prm, a, b, w, h, ma, mb, want_reasons=True)
    runs = [(flags, "auto") for flags in paths]
    if prm.cost_mode == 0 and prm.aggregate_bytes == 2:  # compact SGM: Census, 16-bit
        runs.append((0, "esgm"))
    for flags, mode in runs:
        prm.flags = flags
        session.set_streaming(mode)
        try:
            got = session.pair(prm, a, b, w, h, ma, mb, want_views=True, want_reasons=True)
        finally:
            session.set_streaming("auto")
        what = (flags, mode)
        assert np.array_equal(bits(got.left), bits(want["dl"])), what
        assert np.array_equal(bits(got.right), bits(want["dr"])), what
        assert np.array_equal(bits(got.disparity), bits(want["checked"])), what
        assert np.array_equal(got.reasons, want["reasons"]), what
        assert np.array_equal(got.searchBoundary, want["boundary"]), what
    return want


def noise_pair(w, h, shift, seed):
    rng = np.random.default_rng(seed)
    a = rng.integers(0, 256, (h, w), dtype=np.uint8)
    b = np.roll(a, -shift, axis=1)
    return a.reshape(-1), np.ascontiguousarray(b).reshape(-1)


@pytest.mark.parametrize("census", [3, 5, 11])
def test_smallest_image(session, census):
    w = h = census + 2
    a, b = noise_pair(w, h, 1, census)
    o = Options()
    o.census, o.disparities = census, 3
    check(session, o, a, b, w, h)


@pytest.mark.parametrize("D", [3, 63, 64, 65, 255, 256, 257, 700])
def test_disparity_counts_at_the_kernel_edges(session, D):
    a, b = noise_pair(97, 41, 5, D)
    o = Options()
    o.census, o.disparities, o.minDisparity = 5, D, -2
    check(session, o, a, b, 97, 41)


def test_largest_disparity_count(session):
    """D = 4096 (Options.java: --disparities 3..4096) on a narrow pair: general kernels."""
    a, b = noise_pair(160, 20, 30, 1)
    o = Options()
    o.census, o.disparities, o.minDisparity = 5, 4096, -4000
    check(session, o, a, b, 160, 20)


def test_everything_masked(session):
    a, b = noise_pair(96, 40, 4, 2)
    zero = np.zeros(96 * 40, np.uint8)
    o = Options()
    o.census, o.disparities = 5, 16
    want = check(session, o, a, b, 96, 40, zero, zero)
    assert not np.isfinite(want["checked"]).any() and want["stats"].selected == 0


@pytest.mark.parametrize("w,h", [(131, 29), (130, 30), (67, 65), (1025, 17)])
def test_odd_sizes(session, w, h):
    a, b = noise_pair(w, h, 3, w + h)
    o = Options()
    o.census, o.disparities, o.directions = 5, 24, 8
    check(session, o, a, b, w, h)


def test_taller_than_the_fused_row_limit(session):
    """70000 rows: beyond the fused sweep's 65535, the default path runs the general kernels."""
    a, b = noise_pair(9, 70000, 1, 3)
    o = Options()
    o.census, o.disparities, o.directions = 5, 4, 4
    check(session, o, a, b, 9, 70000, paths=(0,))
