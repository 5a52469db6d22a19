"""Seeded synthetic rectified pairs that stand in for real imagery in the benchmark workloads.

A pair: the left image is seeded uniform noise in [0, 255], Gaussian-blurred (sigma 1.5) and
requantised to the full uint8 range; the right image is the left warped by a ground-truth
disparity field of slanted planes (optionally plus a smooth sinusoid), with disoccluded pixels
filled by fresh noise and i.i.d. Gaussian sensor noise added.  Optional saturated specular
patches.  Everything is vectorised numpy and depends only on the seed.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class PairSpec:
    width: int
    height: int
    planes: int
    d_min: float
    d_max: float
    sinusoid: float = 0.0     # amplitude in px of the smooth height term
    specular: float = 0.0     # fraction of pixels covered by saturated 5x5 patches
    sensor_sigma: float = 2.0
    blur_sigma: float = 1.5
    seed: int = 0


# The benchmark's workloads (sizes, disparity ranges and textures of the stated configurations).
CFG0 = PairSpec(640, 480, planes=3, d_min=4, d_max=60, seed=1000)
CFG1 = PairSpec(1600, 1067, planes=6, d_min=0, d_max=127, sinusoid=8.0, seed=1001)
CFG2 = PairSpec(3000, 2000, planes=10, d_min=0, d_max=255, specular=0.02, seed=1002)


def _gaussian_blur(img: np.ndarray, sigma: float) -> np.ndarray:
    r = int(np.ceil(3 * sigma))
    t = np.arange(-r, r + 1, dtype=np.float64)
    k = np.exp(-0.5 * (t / sigma) ** 2)
    k /= k.sum()
    pad = np.pad(img, r, mode="reflect")
    tmp = sum(k[i] * pad[:, i:i + img.shape[1]] for i in range(2 * r + 1))
    return sum(k[i] * tmp[i:i + img.shape[0], :] for i in range(2 * r + 1))


def _texture(rng: np.random.Generator, h: int, w: int, sigma: float) -> np.ndarray:
    noise = rng.uniform(0, 255, size=(h, w))
    blurred = _gaussian_blur(noise, sigma)
    lo, hi = blurred.min(), blurred.max()
    return np.clip(np.rint((blurred - lo) * (255.0 / max(hi - lo, 1e-9))), 0, 255)


def disparity_field(spec: PairSpec, rng: np.random.Generator) -> np.ndarray:
    """Piecewise-linear field: `planes` slanted planes on a Voronoi partition of the image."""
    h, w = spec.height, spec.width
    ys, xs = np.mgrid[0:h, 0:w].astype(np.float64)
    centers = rng.uniform([0, 0], [w, h], size=(spec.planes, 2))
    dist = (xs[None] - centers[:, 0, None, None]) ** 2 + (ys[None] - centers[:, 1, None, None]) ** 2
    label = dist.argmin(axis=0)
    span = spec.d_max - spec.d_min
    d = np.empty((h, w))
    for i in range(spec.planes):
        base = rng.uniform(spec.d_min + 0.15 * span, spec.d_max - 0.15 * span)
        gx = rng.uniform(-0.25, 0.25) * span / w
        gy = rng.uniform(-0.25, 0.25) * span / h
        m = label == i
        d[m] = base + gx * (xs[m] - centers[i, 0]) + gy * (ys[m] - centers[i, 1])
    if spec.sinusoid:
        d += spec.sinusoid * np.sin(2 * np.pi * xs / (w / 3.0)) * np.cos(2 * np.pi * ys / (h / 2.0))
    return np.clip(d, spec.d_min, spec.d_max)


def make_pair(spec: PairSpec):
    """Returns (left uint8[h*w], right uint8[h*w], disparity float32[h*w] in left coordinates)."""
    rng = np.random.default_rng(spec.seed)
    h, w = spec.height, spec.width
    left = _texture(rng, h, w, spec.blur_sigma)
    d = disparity_field(spec, rng)
    if spec.specular:
        count = int(spec.specular * h * w / 25)
        cy = rng.integers(0, h - 5, count)
        cx = rng.integers(0, w - 5, count)
        for dy in range(5):
            for dx in range(5):
                left[cy + dy, cx + dx] = 255
    # Forward warp with a z-buffer: left (x, y) lands at right (round(x - d), y); nearer
    # (larger d) wins.  Key = quantised d and source column, so the max keeps both.
    xs = np.arange(w)[None, :].repeat(h, 0)
    target = np.rint(xs - d).astype(np.int64)
    ok = (target >= 0) & (target < w)
    rows = np.arange(h)[:, None].repeat(w, 1)
    key = np.full(h * w, -1, np.int64)
    dq = np.rint(d * 256).astype(np.int64)
    flat = (rows * w + np.clip(target, 0, w - 1))[ok]
    np.maximum.at(key, flat, (dq << 13 | xs)[ok])
    right = _texture(rng, h, w, spec.blur_sigma).reshape(-1)  # fresh noise for disocclusions
    hit = key >= 0
    src = (np.arange(h * w) // w) * w + (key & 8191)
    right[hit] = left.reshape(-1)[src[hit]]
    right = right.reshape(h, w)
    left = np.clip(np.rint(left + rng.normal(0, spec.sensor_sigma, size=(h, w))), 0, 255)
    right = np.clip(np.rint(right + rng.normal(0, spec.sensor_sigma, size=(h, w))), 0, 255)
    return (left.astype(np.uint8).reshape(-1), right.astype(np.uint8).reshape(-1),
            d.astype(np.float32).reshape(-1))


def make_color_pair(spec: PairSpec):
    """A rectified colour pair for --census-mode color-distance: three independently textured
    channels, warped by one disparity field as in make_pair, interleaved BGR, with the gray images
    the matcher's costs and penalties read ((29 B + 150 G + 77 R + 128) >> 8).  Returns
    (left gray, right gray, left BGR uint8[h*w*3], right BGR, disparity float32[h*w])."""
    rng = np.random.default_rng(spec.seed)
    h, w = spec.height, spec.width
    left = np.stack([_texture(rng, h, w, spec.blur_sigma) for _ in range(3)], axis=-1)
    d = disparity_field(spec, rng)
    xs = np.arange(w)[None, :].repeat(h, 0)
    target = np.rint(xs - d).astype(np.int64)
    ok = (target >= 0) & (target < w)
    rows = np.arange(h)[:, None].repeat(w, 1)
    key = np.full(h * w, -1, np.int64)
    dq = np.rint(d * 256).astype(np.int64)
    flat = (rows * w + np.clip(target, 0, w - 1))[ok]
    np.maximum.at(key, flat, (dq << 13 | xs)[ok])
    hit = key >= 0
    src = (np.arange(h * w) // w) * w + (key & 8191)
    right = np.stack([_texture(rng, h, w, spec.blur_sigma) for _ in range(3)], axis=-1)
    right = right.reshape(-1, 3)
    right[hit] = left.reshape(-1, 3)[src[hit]]
    right = right.reshape(h, w, 3)
    left = np.clip(np.rint(left + rng.normal(0, spec.sensor_sigma, size=left.shape)), 0, 255)
    right = np.clip(np.rint(right + rng.normal(0, spec.sensor_sigma, size=right.shape)), 0, 255)
    left, right = left.astype(np.uint8), right.astype(np.uint8)

    def gray(bgr):
        b, g, r = (bgr[..., i].astype(np.int32) for i in range(3))
        return ((29 * b + 150 * g + 77 * r + 128) >> 8).astype(np.uint8).reshape(-1)

    return (gray(left), gray(right), left.reshape(-1), right.reshape(-1),
            d.astype(np.float32).reshape(-1))


def spec_for(name: str, seed_offset: int = 0) -> PairSpec:
    base = {"cfg0": CFG0, "cfg1": CFG1, "cfg2": CFG2}[name]
    return PairSpec(**{**base.__dict__, "seed": base.seed + seed_offset})
