"""The host census of pose_b200.census_host equals the oracle's CensusSgm.census / textureMask
restatement bit for bit (square windows of the reference and the 9x7 extension)."""
from __future__ import annotations

import numpy as np
import pytest

from pose_b200 import census_host


@pytest.mark.parametrize("wx,wy", [(3, 3), (5, 5), (9, 7), (9, 9), (11, 11)])
def test_host_census_equals_oracle(oracle_lib, wx, wy):
    rng = np.random.default_rng(wx * 16 + wy)
    w, h = 97, 41
    img = rng.integers(0, 256, w * h, dtype=np.uint8)
    img[: w * 3] = 128  # a flat band: untextured pixels
    assert np.array_equal(census_host.census(img, w, h, wx, wy),
                          oracle_lib.census(img, w, h, wx, wy))
    assert np.array_equal(census_host.texture(img, w, h, wx, wy),
                          oracle_lib.texture(img, w, h, wx, wy))
