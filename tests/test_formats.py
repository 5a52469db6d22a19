"""Disparity PFM (DenseReconstruction.java:943-956) and stereo cache payload
(ReuseCache.java:198-203, 235-240, 557-621) byte layouts.

The expected bytes are assembled here field by field from the reference's writer code, not by
the functions under test."""
from __future__ import annotations

import struct

import numpy as np
import pytest

from pose_b200 import formats
from pose_b200.sgm import Stats


def test_pfm_bytes_and_round_trip(tmp_path):
    d = np.array([1.5, -0.0, np.nan, 2.25, 3.0, np.inf], np.float32)  # 3 x 2, row-major
    path = tmp_path / "d.pfm"
    formats.write_disparity_pfm(path, 3, 2, d)
    want = b"Pf\n3 2\n-1.0\n" + struct.pack("<3f", 2.25, 3.0, np.inf) + \
        struct.pack("<3f", 1.5, -0.0, np.nan)
    assert path.read_bytes() == want
    w, h, back = formats.read_disparity_pfm(path)
    assert (w, h) == (3, 2)
    assert np.array_equal(back.view(np.uint32), d.view(np.uint32))


def test_stereo_payload_bytes():
    stats = Stats()
    stats.selected, stats.valid, stats.speckleRejected = 7, 5, 2
    d = np.array([0.5, np.nan], np.float32)
    data = formats.stereo_payload(2, 1, stats, d, None, np.array([0.25, 1.0], np.float32))
    counters = [0, 0, 0, 0, 0, 0, 0, 0, 7, 0, 0, 0, 2, 5]
    want = struct.pack(">iii", 0x53474D32, 2, 1) + struct.pack(">14q", *counters) + \
        struct.pack(">i2f", 2, 0.5, np.nan) + struct.pack(">i", -1) + \
        struct.pack(">i2f", 2, 0.25, 1.0)
    assert data == want
    got, disp, corr, lr = formats.read_stereo_payload(data, 2, 1)
    assert got["selected"] == 7 and got["valid"] == 5 and got["speckleRejected"] == 2
    assert corr is None
    assert np.array_equal(disp.view(np.uint32), d.view(np.uint32))
    assert np.array_equal(lr, np.array([0.25, 1.0], np.float32))


@pytest.mark.parametrize("mutate,message", [
    (lambda b: struct.pack(">i", 0x53474D31) + b[4:], "Unknown cache version"),
    (lambda b: b + b"\0", "Trailing cache bytes"),
    (lambda b: b[:-1], "truncated"),
])
def test_stereo_payload_rejects_what_the_reference_rejects(mutate, message):
    data = formats.stereo_payload(2, 1, Stats(), np.zeros(2, np.float32))
    with pytest.raises(ValueError, match=message):
        formats.read_stereo_payload(mutate(data), 2, 1)
    with pytest.raises(ValueError, match="dimension mismatch"):
        formats.read_stereo_payload(data, 1, 2)
