"""Independent restatement of CensusSgm.computeRecorded's post-filters and of colorCensus
(test infrastructure).

Follows src/main/java/sgm/CensusSgm.java:203-272 with the helpers medianValid /
medianEdgePreserving (:557-601), reciprocal (:604-612), zncc (:615-644) and removeSpeckles
(:647-681), one gray channel, and colorCensus (:302-332).  Written from the Java source in plain
Python, apart from the C oracle (oracle/sgm_oracle.c): the median sorts with Python's sorted(),
the speckles are found by a depth-first walk instead of the oracle's queue, and FP64 follows
Python floats (IEEE double, no fused operations) in the Java evaluation order.  Small images
only.
"""
from __future__ import annotations

import math

import numpy as np


def _fsub(a, b) -> float:
    return float(np.float32(a) - np.float32(b))


def _java_round_float(v) -> int:
    # Math.round(float): floor(v + 1/2), exact in double for a float v.
    return math.floor(float(np.float32(v)) + 0.5)


def _window(w, h, x, y, r):
    return range(max(0, y - r), min(h - 1, y + r) + 1), range(max(0, x - r), min(w - 1, x + r) + 1)


def median_valid(a, w, h, window):
    r = window // 2
    out = a.copy()
    for y in range(h):
        for x in range(w):
            if not math.isfinite(a[y * w + x]):
                continue
            ys, xs = _window(w, h, x, y, r)
            values = sorted(float(a[yy * w + xx]) for yy in ys for xx in xs
                            if math.isfinite(a[yy * w + xx]))
            out[y * w + x] = values[len(values) // 2]
    return out


def median_edge_preserving(a, w, h, window, max_change, gray, edge):
    r = window // 2
    out = median_valid(a, w, h, window)
    for y in range(h):
        for x in range(w):
            center = float(a[y * w + x])
            if not math.isfinite(center):
                continue
            if abs(_fsub(out[y * w + x], center)) < max_change:
                continue
            ys, xs = _window(w, h, x, y, r)
            values = sorted(
                float(a[yy * w + xx]) for yy in ys for xx in xs
                if math.isfinite(a[yy * w + xx]) and abs(_fsub(a[yy * w + xx], center)) <= max_change
                and (edge == 0 or abs(int(gray[yy * w + xx]) - int(gray[y * w + x])) <= edge))
            if values:
                out[y * w + x] = values[len(values) // 2]
    return out


def reciprocal(right, w, h, x, y, d, tolerance, border):
    if not math.isfinite(d) or y < border or y >= h - border:
        return False
    xr = _java_round_float(_fsub(float(x), d))
    if xr < border or xr >= w - border:
        return False
    other = float(right[y * w + xr])
    return math.isfinite(other) and abs(_fsub(d, other)) <= tolerance


def zncc(a, b, w, h, x, y, d, r, channels=1):
    target = x - float(d)
    bx = math.floor(target)
    fraction = target - bx
    if x - r < 0 or x + r >= w or y - r < 0 or y + r >= h or bx - r < 0 or bx + r + 1 >= w:
        return -1.0
    n = (2 * r + 1) * (2 * r + 1)
    covariance = var_a = var_b = 0.0
    for channel in range(channels):
        sa = sb = saa = sbb = sab = 0.0
        for dy in range(-r, r + 1):
            for dx in range(-r, r + 1):
                av = float(a[((y + dy) * w + x + dx) * channels + channel])
                bi = ((y + dy) * w + bx + dx) * channels + channel
                bv = (1 - fraction) * float(b[bi]) + fraction * float(b[bi + channels])
                sa += av
                sb += bv
                saa += av * av
                sbb += bv * bv
                sab += av * bv
        covariance += sab - sa * sb / n
        var_a += saa - sa * sa / n
        var_b += sbb - sb * sb / n
    if var_a < channels * n * 4 or var_b < channels * n * 4:
        return -1.0
    product = var_a * var_b
    return covariance / math.sqrt(product if product > 1e-12 else 1e-12)


def remove_speckles(a, w, h, minimum, rng, connectivity):
    if minimum <= 1:
        return 0
    seen = np.zeros(w * h, bool)
    steps = [(1, 0), (-1, 0), (0, 1), (0, -1)]
    if connectivity == 8:
        steps += [(1, 1), (1, -1), (-1, 1), (-1, -1)]
    rejected = 0
    for start in range(w * h):
        if seen[start] or not math.isfinite(a[start]):
            continue
        seen[start] = True
        stack, members = [start], [start]
        while stack:
            p = stack.pop()
            x, y = p % w, p // w
            for dx, dy in steps:
                xx, yy = x + dx, y + dy
                if not (0 <= xx < w and 0 <= yy < h):
                    continue
                q = yy * w + xx
                if seen[q] or not math.isfinite(a[q]) or abs(_fsub(a[q], a[p])) > rng:
                    continue
                seen[q] = True
                stack.append(q)
                members.append(q)
        if len(members) < minimum:
            for q in members:
                a[q] = np.nan
            rejected += len(members)
    return rejected


def postfilter(post, left, right, dr, w, h, checked, counts, reasons, left_bgr=None,
               right_bgr=None):
    """In place on checked (float32) and reasons (uint8); counts is a dict with the four
    counters (postMedianLrRejected and photometricRejected added to, speckleRejected set, valid
    added to).  With the BGR images the gate correlates their three channels."""
    photo_l, photo_r, channels = (left, right, 1) if left_bgr is None else (left_bgr, right_bgr, 3)
    if post["median"] > 1:
        filtered = (median_valid(checked, w, h, post["median"]) if post["classic"] else
                    median_edge_preserving(checked, w, h, post["median"], post["max_change"], left,
                                           post["edge"]))
        checked[:] = filtered
    for y in range(h):
        for x in range(w):
            p = y * w + x
            d = float(checked[p])
            if not math.isfinite(d):
                continue
            if not reciprocal(dr, w, h, x, y, d, post["lr"], post["border"]):
                checked[p] = np.nan
                counts["postMedianLrRejected"] += 1
                reasons[p] = 5
                continue
            if zncc(photo_l, photo_r, w, h, x, y, d, post["window"] // 2,
                    channels) < post["correlation"]:
                checked[p] = np.nan
                counts["photometricRejected"] += 1
                reasons[p] = 6
    before = checked.copy()
    counts["speckleRejected"] = remove_speckles(checked, w, h, post["speckle"], post["range"],
                                                post["connectivity"])
    counts["valid"] += int(np.isfinite(checked).sum())
    reasons[np.isfinite(before) & ~np.isfinite(checked)] = 7


def color_census(bgr, w, h, wx, wy):
    """CensusSgm.colorCensus (CensusSgm.java:302-332), generalised to wx x wy windows with the
    same bit order: (descriptors uint64 [words][w*h], textured bool [w*h])."""
    rx, ry = wx // 2, wy // 2
    words = (wx * wy - 1 + 63) // 64
    desc = np.zeros((words, w * h), np.uint64)
    tex = np.zeros(w * h, bool)
    img = np.asarray(bgr, np.int64).reshape(h, w, 3)
    for y in range(ry, h - ry):
        for x in range(rx, w - rx):
            distances = []
            for dy in range(-ry, ry + 1):
                for dx in range(-rx, rx + 1):
                    if dx == 0 and dy == 0:
                        continue
                    squared = 0.0
                    for c in range(3):
                        diff = int(img[y + dy, x + dx, c]) - int(img[y, x, c])
                        squared += float(diff * diff)
                    distances.append(math.sqrt(squared))
            total = 0.0
            for value in distances:
                total += value
            mean = total / (wx * wy)  # the centre's zero distance counts in the mean
            tex[y * w + x] = max(distances) >= 4
            for k, value in enumerate(distances):
                if value >= mean:
                    desc[k // 64, y * w + x] |= np.uint64(1 << (k % 64))
    return desc, tex
