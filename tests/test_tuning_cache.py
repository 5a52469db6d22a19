"""The autotuner's cache file, read without a device (csgm_tuning_cache_lookup): buckets by
padded disparity count, paths and half-octave width / height; malformed lines are skipped."""
from __future__ import annotations

import ctypes

import pytest

from pose_b200 import _abi
from pose_b200.options import Options
from pose_b200.stereo_cost import params_from_options


@pytest.fixture(scope="module")
def lib():
    from pose_b200 import build

    build.build()
    return _abi.load()


def lookup(lib, path, prm, w, h):
    t = _abi.CsgmTuning()
    _abi.check(lib.csgm_tuning_cache_lookup(str(path).encode(), ctypes.byref(prm), w, h,
                                            ctypes.byref(t)))
    return t


def test_cache_lookup_buckets(lib, tmp_path):
    path = tmp_path / "tuning.txt"
    # 1600 -> round(2 log2 1600) = 21, 1067 -> 20; 640 -> 19, 480 -> 18
    path.write_text(
        "csgm-tuning v1 dp=128 paths=8 wb=21 hb=20 rows=8 line_warps=4 line_slack=150 ms=3.5\n"
        "garbage line\n"
        "csgm-tuning v1 dp=64 paths=8 wb=19 hb=18 rows=4 line_warps=0 line_slack=100 ms=0.4\n")
    o = Options()
    o.disparities = 128
    prm = params_from_options(o)
    t = lookup(lib, path, prm, 1600, 1067)
    assert (t.rows_per_block, t.line_warps, t.line_slack, t.disparity_lanes) == (8, 4, 150, 4)
    assert t.milliseconds == pytest.approx(3.5)
    assert lookup(lib, path, prm, 1700, 1000).rows_per_block == 8  # same half-octave buckets
    assert lookup(lib, path, prm, 3000, 2000).rows_per_block == 0  # no entry
    o.disparities = 40  # padded to 64
    t = lookup(lib, path, params_from_options(o), 640, 480)
    assert (t.rows_per_block, t.line_warps, t.disparity_lanes) == (4, 0, 2)
    o.directions = 4
    assert lookup(lib, path, params_from_options(o), 640, 480).rows_per_block == 0


def test_missing_cache_is_empty(lib, tmp_path):
    prm = params_from_options(Options())
    assert lookup(lib, tmp_path / "absent.txt", prm, 640, 480).rows_per_block == 0
