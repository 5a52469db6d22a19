"""The autotuner on the GPU: csgm_autotune times the sweep's launch shapes, keeps the fastest per
bucket and caches it; a fresh session loads the cache; every shape gives the same bits."""
from __future__ import annotations

import numpy as np
import pytest

import oracle.oracle as orc
from pose_b200 import _abi
from pose_b200.options import Options
from pose_b200.stereo_cost import params_from_options

pytestmark = pytest.mark.gpu


def params(D=64, directions=8):
    o = Options()
    o.census, o.censusHeight, o.disparities, o.directions = 9, 7, D, directions
    prm = params_from_options(o)
    prm.p1, prm.p2 = 10, 120
    return prm


def test_autotune_caches_and_reloads(tmp_path):
    from pose_b200.sgm import GpuSgm

    cache = str(tmp_path / "tuning.txt")
    prm = params(D=128)
    w, h = 800, 534
    with GpuSgm(0) as s:
        best = s.autotune(prm, w, h, cache)
        assert best["rows_per_block"] in (4, 8, 12) and best["line_warps"] in (0, 4, 8)
        assert best["disparity_lanes"] == 4 and best["milliseconds"] > 0
        assert s.tuning(prm, w, h) == best
        other = s.autotune(params(D=64, directions=4), 640, 480, cache)
        assert other["line_warps"] == 0
    lines = open(cache).read().splitlines()
    assert len(lines) == 2 and all(line.startswith("csgm-tuning v1 ") for line in lines)
    with GpuSgm(0) as s:
        default = s.tuning(prm, w, h)
        assert default["milliseconds"] == 0
        s.load_tuning(cache)
        again = s.tuning(prm, w, h)
        assert again["milliseconds"] == pytest.approx(best["milliseconds"], abs=1e-5)
        again.pop("milliseconds")
        best.pop("milliseconds")
        assert again == best


@pytest.mark.parametrize("D,directions", [(128, 8), (256, 8), (256, 16), (192, 4)])
def test_every_launch_shape_gives_the_same_bits(D, directions):
    """A pair under each shape the autotuner tries, forced, against the oracle."""
    from pose_b200.sgm import GpuSgm
    from pose_b200.synthetic import PairSpec, make_pair

    spec = PairSpec(400, 140, planes=3, d_min=4, d_max=100, seed=9)
    left, right, _ = make_pair(spec)
    w, h = spec.width, spec.height
    prm = params(D=D, directions=directions)
    want = orc.pair(prm, left, right, w, h, want_reasons=True)
    regs = (D + 63) // 64 * 2
    with GpuSgm(0) as s:
        for rows in (4, 8, 12) if regs == 4 else (4, 8):
            for lw in (0, 4, 8):
                for slack in (10, 100, 400):
                    s.set_tuning({"rows_per_block": rows, "line_warps": lw, "line_slack": slack})
                    t = s.tuning(prm, w, h)
                    if directions < 8 or (lw and t["line_warps"] != lw):
                        # no line warps in 4-path mode; shapes whose line rings exceed a CTA's
                        # shared memory run with fewer line warps
                        assert t["line_warps"] < max(lw, 1)
                    else:
                        assert (t["rows_per_block"], t["line_warps"], t["line_slack"]) == (
                            rows, lw, slack)
                    got = s.pair(prm, left, right, w, h, want_views=True, want_reasons=True)
                    assert np.array_equal(got.disparity.view(np.uint32),
                                          want["checked"].view(np.uint32)), (rows, lw, slack)
                    assert np.array_equal(got.right.view(np.uint32), want["dr"].view(np.uint32))
        s.set_tuning(None)


def test_autotune_refuses_general_parameters(tmp_path):
    from pose_b200.sgm import GpuSgm

    prm = params(D=300)  # beyond the fused kernels
    with GpuSgm(0) as s:
        with pytest.raises(_abi.CsgmError) as e:
            s.autotune(prm, 640, 480, str(tmp_path / "t.txt"))
        assert e.value.status == _abi.CSGM_E_UNSUPPORTED
