"""The pyramid matcher in front of the stereo matcher: DenseMatcher.compute
(src/main/java/sgm/DenseMatcher.java:10-101) with its refinement (:103-275), tile (:290-351),
crop (:353-369) and resize (:371-384).

A coarse level matches the whole downscaled pair over the full (scaled) disparity range; each
finer level matches overlapping tiles whose disparity range is predicted from the level below
(the sampled disparities plus or minus ``pyramidRadius``), falling back to the full range where a
tile's prediction leaves too many boundary rejections or too few valid pixels.  Every match is
``CensusSgm.computeRecorded`` on the GPU (csgm_pair and csgm_postfilter); the tiling, range
prediction, resizing and counters are host logic, as in the reference.  The reference calls the
result exact inside each tile and a local approximation across tiles; the same holds here.

Resizing is OpenCV's ``cv::resize`` (OpenCV 4.9.0, the reference's pinned dependency, absent
from it): INTER_AREA for images and INTER_NEAREST for masks.  ``resize_area`` restates the area
algorithm: an integer factor averages each factor x factor block (2 x 2 with integer rounding
(sum + 2) >> 2, others the sum times 1/area in float32, rounded to nearest even); a fractional
factor weights the source pixels by their overlap with the destination pixel (weights in
float32, from the interval arithmetic in float64), summing each source row's weighted pixels in
order and then the weighted rows in order, in float32, rounded to nearest even and saturated.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from .sgm import Result, Stats


def _java_round(v: float) -> int:
    f = math.floor(v)
    return int(f + 1 if v - f >= 0.5 else f)


def _area_tab(ssize: int, dsize: int, scale: float):
    """Per destination index, the (source index, float32 weight) pairs of its area."""
    per = [[] for _ in range(dsize)]
    for dx in range(dsize):
        f1 = dx * scale
        f2 = f1 + scale
        cell = min(scale, ssize - f1)
        s1, s2 = math.ceil(f1), math.floor(f2)
        s2 = min(s2, ssize - 1)
        s1 = min(s1, s2)
        if s1 - f1 > 1e-3:
            per[dx].append((s1 - 1, np.float32((s1 - f1) / cell)))
        for sx in range(s1, s2):
            per[dx].append((sx, np.float32(1.0 / cell)))
        if f2 - s2 > 1e-3:
            per[dx].append((s2, np.float32(min(min(f2 - s2, 1.0), cell) / cell)))
    return per


def _weighted(src: np.ndarray, per, dsize: int) -> np.ndarray:
    """out[:, d] = sum over per[d] in order of src[:, s] * weight, in float32."""
    out = np.zeros((src.shape[0], dsize) + src.shape[2:], np.float32)
    for j in range(max(len(p) for p in per)):
        idx = [d for d in range(dsize) if len(per[d]) > j]
        s = np.array([per[d][j][0] for d in idx])
        wgt = np.array([per[d][j][1] for d in idx], np.float32)
        if src.ndim == 3:
            wgt = wgt[:, None]
        out[:, idx] = (out[:, idx] + (src[:, s] * wgt).astype(np.float32)).astype(np.float32)
    return out


def resize_area(img: np.ndarray, width: int, height: int) -> np.ndarray:
    """cv::resize INTER_AREA of an [h, w] or [h, w, c] uint8 image to [height, width(, c)]."""
    h, w = img.shape[:2]
    fx, fy = w / width, h / height
    if abs(fx - round(fx)) < 1e-9 and abs(fy - round(fy)) < 1e-9:
        ix, iy = int(round(fx)), int(round(fy))
        block = img[:height * iy, :width * ix].astype(np.int64)
        block = block.reshape(height, iy, width, ix, *img.shape[2:]).sum(axis=(1, 3))
        if ix == 2 and iy == 2:
            return ((block + 2) >> 2).astype(np.uint8)
        scaled = (block * np.float32(1.0 / (ix * iy))).astype(np.float32)
        return np.clip(np.rint(scaled), 0, 255).astype(np.uint8)
    rows = _weighted(img.astype(np.float32), _area_tab(w, width, fx), width)
    cols = _weighted(np.swapaxes(rows, 0, 1), _area_tab(h, height, fy), height)
    return np.clip(np.rint(np.swapaxes(cols, 0, 1)), 0, 255).astype(np.uint8)


def resize_nearest(img: np.ndarray, width: int, height: int) -> np.ndarray:
    """cv::resize INTER_NEAREST: source index floor(d * size / dsize), clamped."""
    h, w = img.shape[:2]
    xs = np.minimum(np.floor(np.arange(width) * (w / width)).astype(np.int64), w - 1)
    ys = np.minimum(np.floor(np.arange(height) * (h / height)).astype(np.int64), h - 1)
    return img[ys][:, xs]


def resize(data, w: int, h: int, width: int, height: int, channels: int, mask: bool):
    """DenseMatcher.resize (:371-384) on flat row-major buffers."""
    if data is None:
        return None
    if w == width and h == height:
        return data
    img = np.asarray(data, np.uint8).reshape((h, w) if channels == 1 else (h, w, channels))
    out = resize_nearest(img, width, height) if mask else resize_area(img, width, height)
    return np.ascontiguousarray(out).reshape(-1)


def crop(data, w: int, h: int, x: int, y: int, width: int, height: int, channels: int):
    """DenseMatcher.crop (:353-369): zeros outside the image."""
    if data is None:
        return None
    src = np.asarray(data, np.uint8).reshape(h, w * channels)
    out = np.zeros((height, width * channels), np.uint8)
    y0, y1 = max(0, y), min(h, y + height)
    x0, x1 = max(0, x), min(w, x + width)
    if y1 > y0 and x1 > x0:
        out[y0 - y:y1 - y, (x0 - x) * channels:(x1 - x) * channels] = \
            src[y0:y1, x0 * channels:x1 * channels]
    return out.reshape(-1)


def memory_estimate(w: int, h: int, d: int, o) -> int:
    """CensusSgm.memoryEstimate(w, h, d, Options) (CensusSgm.java:276-286)."""
    from .stereo_cost import StereoCost

    words = (o.census * o.census - 1 + 63) // 64
    base = w * h * d * 6 + w * d * 8 + w * h * (48 + 16 * words)
    return base - w * h * d * (4 - StereoCost.aggregateBytes(o))


@dataclass
class _Tile:
    result: Result
    halo: int
    halo_y: int
    minimum: int
    count: int
    valid: int
    boundary: int


class DenseMatcher:
    """DenseMatcher over a stereo backend: ``compute_recorded(options, a, b, ca, cb, w, h, ma,
    mb)`` returns a Result with disparity, stats, reasons and searchBoundary, as
    ``CensusSgm.computeRecorded`` with a collecting observer does (DenseMatcher.java:306-318).
    ``gpu_backend`` gives the GPU one."""

    def __init__(self, compute_recorded):
        self.compute_recorded = compute_recorded

    # DenseMatcher.compute (:10-101)
    def compute(self, o, left, right, color, color_right, w, h, mask_a=None, mask_b=None):
        if o.pyramidLevels == 1:
            return self.compute_recorded(o, left, right, color, color_right, w, h, mask_a, mask_b)
        levels = o.pyramidLevels
        if levels == 0:
            levels = 1
            budget = o.memoryMb * 1048576
            while levels < 6 and min(w, h) // (1 << levels) >= 32:
                factor = 1 << (levels - 1)
                cw, ch = max(1, w // factor), max(1, h // factor)
                cd = max(3, (o.disparities + factor - 1) // factor)
                if cd <= 96 and memory_estimate(cw, ch, cd, o) <= budget:
                    break
                levels += 1
        while levels > 1 and min(w, h) // (1 << (levels - 1)) < 32:
            levels -= 1
        color_mode = o.censusMode == "color-distance"
        previous, pw, ph, result, coarse = None, 0, 0, None, None
        for level in range(levels - 1, -1, -1):
            factor = 1 << level
            lw = max(1, _java_round(w / factor))
            lh = max(1, _java_round(h / factor))
            scale = lw / w
            a = resize(left, w, h, lw, lh, 1, False)
            b = resize(right, w, h, lw, lh, 1, False)
            ma = resize(mask_a, w, h, lw, lh, 1, True)
            mb = resize(mask_b, w, h, lw, lh, 1, True)
            ca = resize(color, w, h, lw, lh, 3, False) if color_mode else None
            cb = resize(color_right, w, h, lw, lh, 3, False) if color_mode else None
            cur = o.copy()
            cur.pyramidLevels = 1
            cur.minDisparity = math.floor(o.minDisparity * scale)
            cur.disparities = max(3, math.ceil((o.minDisparity + o.disparities - 1) * scale)
                                  - cur.minDisparity + 1)
            cur.speckleSize = o.speckleSize if level == 0 else max(0, o.speckleSize
                                                                    // (factor * factor))
            if previous is None:
                result = self.compute_recorded(cur, a, b, ca, cb, lw, lh, ma, mb)
                coarse = result.stats
            else:
                result = self._refine(cur, a, b, ca, cb, lw, lh, ma, mb, previous, pw, ph)
            previous = result.disparity
            if level == 0 and coarse is not None and coarse is not result.stats:
                result.stats.coarseLowerBoundaryRejected = coarse.lowerBoundaryRejected
                result.stats.coarseUpperBoundaryRejected = coarse.upperBoundaryRejected
                result.stats.coarseFullIntervalPixels = coarse.fullIntervalPixels
            pw, ph = lw, lh
        return result

    # DenseMatcher.refine (:103-275)
    def _refine(self, o, a, b, ca, cb, w, h, ma, mb, previous, pw, ph):
        out = np.full(w * h, np.nan, np.float32)
        reasons = np.ones(w * h, np.uint8)
        stats = Stats()
        self.fallbacks = 0
        self.tiles = []
        for y in range(0, h, o.tileSize):
            for x in range(0, w, o.tileSize):
                tw, th = min(o.tileSize, w - x), min(o.tileSize, h - y)
                samples, coverage, potential = [], set(), 0
                for yy in range(y, y + th, 4):
                    for xx in range(x, x + tw, 4):
                        potential += 1
                        v = float(previous[min(ph - 1, int(yy * ph / h)) * pw
                                           + min(pw - 1, int(xx * pw / w))])
                        if math.isfinite(v):
                            samples.append(v * w / pw)
                            coverage.add(min(3, (xx - x) * 4 // max(1, tw))
                                         + 4 * min(3, (yy - y) * 4 // max(1, th)))
                samples.sort()
                lo, hi = o.minDisparity, o.minDisparity + o.disparities - 1
                predicted = len(samples) >= max(8, potential // 5) and len(coverage) >= 4
                if predicted:
                    lo = max(lo, math.floor(samples[0]) - o.pyramidRadius)
                    hi = min(hi, math.ceil(samples[-1]) + o.pyramidRadius)
                t = self._tile(o, a, b, ca, cb, w, h, ma, mb, x, y, tw, th, lo, hi)
                if predicted and (t.boundary > max(16, .01 * tw * th)
                                  or t.valid < max(4, tw * th // 100)):
                    t = self._tile(o, a, b, ca, cb, w, h, ma, mb, x, y, tw, th, o.minDisparity,
                                   o.minDisparity + o.disparities - 1)
                    self.fallbacks += 1
                self.tiles.append({"x": x, "y": y, "width": tw, "height": th,
                                   "prediction_samples": len(samples),
                                   "occupied_cells": len(coverage), "min_disparity": t.minimum,
                                   "disparities": t.count, "valid": t.valid,
                                   "boundary_rejected": t.boundary,
                                   "prediction_used": predicted})
                r, width = t.result, t.result.width
                src = ((np.arange(th)[:, None] + t.halo_y) * width
                       + np.arange(tw)[None, :] + t.halo).reshape(-1)
                dst = ((y + np.arange(th))[:, None] * w + x + np.arange(tw)[None, :]).reshape(-1)
                value = r.disparity[src]
                out[dst] = np.where(np.isfinite(value), value + np.float32(t.minimum), np.nan)
                reasons[dst] = r.reasons[src]
                flags = r.searchBoundary[src]
                stats.fullIntervalPixels += int(((flags & 4) != 0).sum())
                if t.minimum == o.minDisparity:
                    stats.lowerBoundaryRejected += int(((flags & 1) != 0).sum())
                if t.minimum + t.count - 1 == o.minDisparity + o.disparities - 1:
                    stats.upperBoundaryRejected += int(((flags & 2) != 0).sum())
        stats.valid = int(np.isfinite(out).sum())
        stats.boundaryRejected = int((reasons == 2).sum())
        stats.ambiguityRejected = int((reasons == 3).sum())
        stats.lrRejected = int((reasons == 4).sum())
        stats.postMedianLrRejected = int((reasons == 5).sum())
        stats.photometricRejected = int((reasons == 6).sum())
        stats.speckleRejected = int((reasons == 7).sum())
        stats.selected = (stats.valid + stats.lrRejected + stats.postMedianLrRejected
                          + stats.photometricRejected + stats.speckleRejected)
        return Result(w, h, out, stats, reasons=reasons)

    # DenseMatcher.tile (:290-351)
    def _tile(self, o, a, b, ca, cb, w, h, ma, mb, x, y, tw, th, lo, hi):
        count = max(3, hi - lo + 1)
        halo = max(o.tileOverlap, count + o.census + o.correlationWindow + o.median)
        halo_y = max(o.tileOverlap, o.census + o.correlationWindow + o.median)
        width, height = tw + 2 * halo, th + 2 * halo_y
        local = o.copy()
        local.minDisparity = 0
        local.disparities = count
        local.pyramidLevels = 1
        r = self.compute_recorded(
            local, crop(a, w, h, x - halo, y - halo_y, width, height, 1),
            crop(b, w, h, x - halo - lo, y - halo_y, width, height, 1),
            crop(ca, w, h, x - halo, y - halo_y, width, height, 3),
            crop(cb, w, h, x - halo - lo, y - halo_y, width, height, 3), width, height,
            crop(ma, w, h, x - halo, y - halo_y, width, height, 1),
            crop(mb, w, h, x - halo - lo, y - halo_y, width, height, 1))
        at = ((np.arange(th)[:, None] + halo_y) * width + np.arange(tw)[None, :] + halo).reshape(-1)
        valid = int(np.isfinite(r.disparity[at]).sum())
        boundary = int((r.reasons[at] == 2).sum())
        return _Tile(r, halo, halo_y, lo, count, valid, boundary)


def gpu_backend(session):
    """CensusSgm.computeRecorded on the GPU session (csgm_pair / csgm_pair_color, then
    csgm_postfilter / csgm_postfilter_color), with reasons and search-boundary flags."""
    from .sgm import CensusSgm

    def compute_recorded(o, a, b, ca, cb, w, h, ma, mb):
        if (ma is None) != (mb is None):
            raise ValueError("Invalid stereo mask dimensions")
        return CensusSgm(o, session=session).compute(a, b, w, h, ma, mb, want_reasons=True,
                                                     leftBgr=ca, rightBgr=cb)

    return compute_recorded
