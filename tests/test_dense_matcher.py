"""The pyramid matcher (DenseMatcher.java): OpenCV's resize as restated, the reference's own
pyramid regression on the CPU oracle, and (GPU) the CUDA matcher under it against the oracle."""
from __future__ import annotations

import numpy as np
import pytest

from fixtures import storage_gpu_pair
from pose_b200 import dense_matcher as dm
from pose_b200.options import Options
from reference_cpu import compute_recorded_cpu


@pytest.mark.parametrize("w,h,W,H,c", [(64, 48, 32, 24, 1), (65, 47, 33, 24, 1),
                                       (1600, 1067, 800, 534, 1), (1600, 1067, 200, 133, 1),
                                       (99, 77, 50, 39, 3), (641, 481, 80, 60, 1),
                                       (320, 240, 107, 80, 1), (160, 96, 40, 24, 3)])
def test_resize_matches_opencv(w, h, W, H, c):
    """resize_area / resize_nearest equal cv2.resize INTER_AREA / INTER_NEAREST bit for bit
    (OpenCV 4.x; the reference pins 4.9.0)."""
    cv2 = pytest.importorskip("cv2")
    rng = np.random.default_rng(w * 7 + h)
    img = rng.integers(0, 256, (h, w) if c == 1 else (h, w, c), dtype=np.uint8)
    assert np.array_equal(dm.resize_area(img, W, H),
                          cv2.resize(img, (W, H), interpolation=cv2.INTER_AREA))
    assert np.array_equal(dm.resize_nearest(img, W, H),
                          cv2.resize(img, (W, H), interpolation=cv2.INTER_NEAREST))


def test_crop_pads_with_zeros():
    img = np.arange(12, dtype=np.uint8)  # 4 x 3
    out = dm.crop(img, 4, 3, -1, 1, 3, 3, 1).reshape(3, 3)
    assert out.tolist() == [[0, 4, 5], [0, 8, 9], [0, 0, 0]]


def pyramid_options():
    """StorageGpuRegression.java:105-113."""
    o = Options()
    o.disparities, o.pyramidLevels, o.tileSize, o.tileOverlap = 32, 3, 64, 16
    o.pyramidRadius, o.speckleSize = 8, 0
    return o


def shift_error(disp, w, h):
    """StorageGpuRegression.java:124-133: valid pixels and mean |d - 8| of the interior."""
    d = disp.reshape(h, w)[16:h - 16, 20:w - 16]
    ok = np.isfinite(d)
    return int(ok.sum()), float(np.abs(d[ok] - 8).sum() / max(1, ok.sum()))


def test_pyramid_recovers_the_shift_on_the_oracle(oracle_lib):
    """The reference's pyramid regression with the CPU matcher under the pyramid: the
    overlapping tiles recover the eight-pixel shift (valid > 3000, mean error < 0.2)."""
    w, h, a, b, mask = storage_gpu_pair()
    res = dm.DenseMatcher(compute_recorded_cpu).compute(pyramid_options(), a, b, None, None, w,
                                                        h, mask, mask)
    valid, error = shift_error(res.disparity, w, h)
    assert valid > 3000 and error < 0.2, (valid, error)
    assert res.stats.valid == int(np.isfinite(res.disparity).sum())


@pytest.mark.gpu
@pytest.mark.parametrize("levels", [2, 3, 0])
def test_pyramid_gpu_equals_oracle(oracle_lib, levels):
    """StorageGpuRegression.java:114-123: the pyramid over the CUDA matcher equals the pyramid
    over the CPU oracle exactly (tile seams, fallback intervals, counters)."""
    from pose_b200.sgm import GpuSgm

    w, h, a, b, mask = storage_gpu_pair()
    o = pyramid_options()
    o.pyramidLevels = levels
    want = dm.DenseMatcher(compute_recorded_cpu).compute(o, a, b, None, None, w, h, mask, mask)
    with GpuSgm(0) as s:
        got = dm.DenseMatcher(dm.gpu_backend(s)).compute(o, a, b, None, None, w, h, mask, mask)
    assert np.array_equal(got.disparity.view(np.uint32), want.disparity.view(np.uint32))
    assert got.stats.csv() == want.stats.csv()
    valid, error = shift_error(got.disparity, w, h)
    assert valid > 3000 and error < 0.2, (valid, error)


@pytest.mark.gpu
def test_pyramid_color_mode_gpu_equals_oracle(oracle_lib):
    """Colour-distance mode through the pyramid: BGR images resized with INTER_AREA per level."""
    from pose_b200.sgm import GpuSgm
    from pose_b200.synthetic import PairSpec, make_color_pair

    left, right, lbgr, rbgr, _ = make_color_pair(PairSpec(192, 128, planes=3, d_min=6,
                                                          d_max=26, seed=13))
    o = pyramid_options()
    o.censusMode = "color-distance"
    want = dm.DenseMatcher(compute_recorded_cpu).compute(o, left, right, lbgr, rbgr, 192, 128)
    with GpuSgm(0) as s:
        got = dm.DenseMatcher(dm.gpu_backend(s)).compute(o, left, right, lbgr, rbgr, 192, 128)
    assert np.array_equal(got.disparity.view(np.uint32), want.disparity.view(np.uint32))
    assert got.stats.csv() == want.stats.csv()
