"""GPU colour-distance census (csgm_color_census) against the oracle's restatement of
CensusSgm.colorCensus (CensusSgm.java:302-332): descriptors and texture bit for bit."""
from __future__ import annotations

import numpy as np
import pytest

import oracle.oracle as orc

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def session():
    from pose_b200.sgm import GpuSgm

    s = GpuSgm(0)
    yield s
    s.close()


def bgr_image(w, h, seed):
    """Smooth colour ramps with noise, a flat patch (untextured) and a hard edge."""
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:h, 0:w]
    img = np.stack([(xx * 3 + yy) % 256, (yy * 5) % 256, (xx * yy) % 256], -1).astype(np.int32)
    img += rng.integers(-6, 7, img.shape)
    img[h // 4:h // 2, w // 4:w // 2] = (90, 120, 150)
    img[:, (3 * w) // 4:] = 255 - img[:, (3 * w) // 4:]
    return np.clip(img, 0, 255).astype(np.uint8).reshape(-1)


@pytest.mark.parametrize("w,h,seed", [(64, 48, 1), (101, 37, 2)])
@pytest.mark.parametrize("wx,wy", [(3, 3), (5, 5), (9, 7), (9, 9), (11, 11)])
def test_color_census_matches_oracle(session, w, h, seed, wx, wy):
    bgr = bgr_image(w, h, seed)
    want_desc, want_tex = orc.color_census(bgr, w, h, wx, wy)
    desc, tex = session.color_census(bgr, w, h, wx, wy)
    assert np.array_equal(desc.reshape(-1), np.asarray(want_desc).reshape(-1))
    assert np.array_equal(tex.astype(bool), np.asarray(want_tex).astype(bool))
    assert tex.any() and not tex.all()
