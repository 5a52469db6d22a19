"""The reference's stereo fixtures, regenerated exactly (java.util.Random, integer shifts, masks).

Each builder cites the reference test it reproduces.  Options returned are the reference's
``TestSupport.options()`` defaults plus the test's own overrides.
"""
from __future__ import annotations

import math

import numpy as np

from jrandom import JavaRandom
from pose_b200.options import Options


def shifted(a: np.ndarray, w: int, h: int, shift: int) -> np.ndarray:
    """b[y*w+x] = a[y*w + min(w-1, x+shift)]."""
    img = a.reshape(h, w)
    cols = np.minimum(np.arange(w) + shift, w - 1)
    return np.ascontiguousarray(img[:, cols]).reshape(-1)


def selftest_pair():
    """src/test/java/sgm/SelfTest.java:82-86: 96x48, Random(4), right = left shifted by 6."""
    w, h = 96, 48
    left = JavaRandom(4).nextBytes(w * h)
    return w, h, left, shifted(left, w, h, 6)


def selftest_options() -> Options:
    """SelfTest.java:87-91 on top of TestSupport.options()."""
    o = Options()
    o.disparities = 16
    o.census = 5
    o.median = 1
    o.uniqueness = 0.02
    return o


def storage_gpu_pair():
    """src/test/java/sgm/StorageGpuRegression.java:53-61: 160x96, Random(124), shift 8, mask hole."""
    w, h = 160, 96
    a = JavaRandom(124).nextBytes(w * h)
    b = shifted(a, w, h, 8)
    mask = np.full(w * h, 255, np.uint8).reshape(h, w)
    mask[21:60, 71:84] = 0
    return w, h, a, b, mask.reshape(-1)


def scaling_pair():
    """src/test/java/sgm/ScalingRegression.java:43-50: 160x47, Random(219), shift 11, hole in ma."""
    w, h = 160, 47
    a = JavaRandom(219).nextBytes(w * h)
    b = shifted(a, w, h, 11)
    ma = np.full((h, w), 255, np.uint8)
    mb = np.full((h, w), 255, np.uint8)
    ma[10:20, 23:32] = 0
    return w, h, a, b, ma.reshape(-1), mb.reshape(-1)


def upgrade_pair():
    """src/test/java/sgm/UpgradeStereoRegression.java:22-32: 192x79, Random(120), shift 13,
    holes in both masks."""
    w, h, shift = 192, 79, 13
    a = JavaRandom(120).nextBytes(w * h)
    b = shifted(a, w, h, shift)
    ma = np.full((h, w), 255, np.uint8)
    mb = np.full((h, w), 255, np.uint8)
    ma[21:55, 86:97] = 0
    mb[6:18, 53:59] = 0
    return w, h, shift, a, b, ma.reshape(-1), mb.reshape(-1)


def upgrade_large_pair():
    """UpgradeStereoRegression.java:99-103: 800x64, Random(93), shift 130, D=693."""
    ww, hh = 800, 64
    first = JavaRandom(93).nextBytes(ww * hh)
    return ww, hh, first, shifted(first, ww, hh, 130)


def large_gpu_pair():
    """src/test/java/sgm/LargeGpuRegression.java:12-25: 900x1600, Random(34), shift 130, D=693."""
    w, h = 900, 1600
    a = JavaRandom(34).nextBytes(w * h)
    return w, h, a, shifted(a, w, h, 130)


def texture(x: float, y: float) -> int:
    """src/test/java/sgm/SubpixelRegression.java:38-46 (Java Math.sin/cos; the last-ulp
    difference of C's libm can flip a rounding, which the thresholds tolerate)."""
    v = (128 + 27 * math.sin(.71 * x + .23 * y) + 23 * math.cos(.43 * x - .69 * y)
         + 21 * math.sin(.29 * x + .91 * y) + 14 * math.cos(1.11 * x + .17 * y))
    c = max(0.0, min(255.0, v))
    f = math.floor(c)
    return int(f + 1 if c - f >= 0.5 else f)


def plane_pair(d: float = 13.37):
    """SubpixelRegression.java:12-19 / MatchingCostBenchmark.java:9-16: 384x192 continuous plane."""
    w, h = 384, 192
    a = np.empty(w * h, np.uint8)
    b = np.empty(w * h, np.uint8)
    for y in range(h):
        for x in range(w):
            a[y * w + x] = texture(x, y)
            b[y * w + x] = texture(x + d, y)
    return w, h, a, b


def plane_metrics(disp: np.ndarray, w: int, h: int, truth: float):
    """SubpixelRegression.metrics (SubpixelRegression.java:48-66)."""
    d = disp.reshape(h, w)[12:h - 12, 45:w - 12].astype(np.float64)
    e = d[np.isfinite(d)] - truth
    e.sort()
    return len(e), math.sqrt(float(np.sum(e * e)) / len(e)), e[len(e) * 9 // 10] - e[len(e) // 10]


def esgm_production_pair(fixture: int):
    """src/test/java/sgm/EsgmProductionRegression.java:15-29: 160x47, Random(174) (fixture 0 and
    2) or a periodic pattern (fixture 1), right = left shifted by 11 (-11 for fixture 2) with the
    column clamped to the image, a 7x5 hole in the left mask."""
    w, h = 160, 47
    a = JavaRandom(174).nextBytes(w * h)
    if fixture == 1:
        y, x = np.mgrid[0:h, 0:w]
        a = ((x % 12) * 19 + (y % 3) * 7).astype(np.uint8).reshape(-1)
    shift = -11 if fixture == 2 else 11
    cols = np.clip(np.arange(w) + shift, 0, w - 1)
    b = np.ascontiguousarray(a.reshape(h, w)[:, cols]).reshape(-1)
    ma = np.full((h, w), 255, np.uint8)
    ma[8:13, 29:36] = 0
    return w, h, a, b, ma.reshape(-1), np.full(w * h, 255, np.uint8)
