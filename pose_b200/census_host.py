"""Census descriptors and texture masks on the host, in the layout csgm_match takes.

The reference computes both on the Java side before it calls GpuSgm.match
(CensusSgm.census, src/main/java/sgm/CensusSgm.java:540-555, and CensusSgm.textureMask,
:523-538): bit k of a pixel's descriptor is set iff the k-th window neighbour (row-major over the
window, centre skipped) is darker than the centre; descriptors are word-major ``[word][pixel]``;
pixels closer than the window radius to an edge keep all-zero descriptors and are untextured;
a pixel is textured when max - min over its window is at least 4.  Rectangular windows use
rx = wx / 2, ry = wy / 2 with the same bit order.  Vectorised numpy; used to prepare inputs of
csgm_match (the GPU path computes its own descriptors in csgm_pair).
"""
from __future__ import annotations

import numpy as np


def words(wx: int, wy: int) -> int:
    """Descriptor words per pixel (CensusSgm.java:519-521)."""
    return (wx * wy - 1 + 63) // 64


def census(img, w: int, h: int, wx: int, wy: int) -> np.ndarray:
    """uint64 [words * w * h] descriptors, word-major."""
    a = np.ascontiguousarray(img, np.uint8).reshape(h, w)
    rx, ry = wx // 2, wy // 2
    out = np.zeros((words(wx, wy), h, w), np.uint64)
    center = a[ry:h - ry, rx:w - rx]
    bit = 0
    for yy in range(-ry, ry + 1):
        for xx in range(-rx, rx + 1):
            if xx == 0 and yy == 0:
                continue
            nb = a[ry + yy:h - ry + yy, rx + xx:w - rx + xx]
            out[bit // 64, ry:h - ry, rx:w - rx] |= (nb < center).astype(np.uint64) << np.uint64(
                bit % 64)
            bit += 1
    return out.reshape(-1)


def texture(img, w: int, h: int, wx: int, wy: int) -> np.ndarray:
    """uint8 [w * h]: 1 where max - min over the window is >= 4 (interior pixels only)."""
    a = np.ascontiguousarray(img, np.uint8).reshape(h, w)
    rx, ry = wx // 2, wy // 2
    lo = np.full((h - 2 * ry, w - 2 * rx), 255, np.uint8)
    hi = np.zeros_like(lo)
    for yy in range(-ry, ry + 1):
        for xx in range(-rx, rx + 1):
            nb = a[ry + yy:h - ry + yy, rx + xx:w - rx + xx]
            np.minimum(lo, nb, out=lo)
            np.maximum(hi, nb, out=hi)
    out = np.zeros((h, w), np.uint8)
    out[ry:h - ry, rx:w - rx] = (hi.astype(np.int16) - lo) >= 4
    return out.reshape(-1)
