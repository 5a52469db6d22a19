"""Stereo-matcher settings: the subset of Collinea's ``Options`` that the SGM path reads.

Field names and defaults follow src/main/java/sgm/Options.java:17-90 (``p1``/``p2`` in 5x5 units,
``census`` window, ``disparities`` ...), and ``validate`` restates the stereo checks of
Options.java:766-933.  One field is an extension: ``censusHeight`` (0 = square window) gives the
rectangular census windows such as 9x7 that the reference does not support.
"""
from __future__ import annotations

import copy
import math
from dataclasses import dataclass


@dataclass
class Options:
    # SGM core (Options.java:17-23, 32, 38-40)
    disparities: int = 128
    minDisparity: int = 0
    census: int = 5
    censusHeight: int = 0  # extension: window height for rectangular census (0 = census)
    directions: int = 8
    p1: float = 4
    p2: float = 24
    uniqueness: float = 0.03
    sgmEdgeScale: int = 32
    matchingCost: str = "census"
    censusWeight: float = 0.5
    adTruncation: int = 30
    gradientTruncation: int = 60
    sgmAggregate: str = "auto"
    censusMode: str = "gray"
    # LR check and post-filters (Options.java:19-22, 67, 76)
    lrThreshold: float = 0.75
    median: int = 3
    medianMode: str = "edge-preserving"
    medianMaxChange: float = 0.5
    medianEdgeThreshold: int = 24
    correlation: float = 0.55
    correlationWindow: int = 7
    speckleSize: int = 50
    speckleRange: float = 1.0
    speckleConnectivity: int = 8
    # device selection (Options.java:90, GpuSgm.java:163-180, 629-633)
    compute: str = "gpu"
    gpuDevice: int = 0
    gpuMemoryMb: int = 0
    # resident, streamed or compact views (Options.java:32,35,39; --gpu-sgm, --esgm-candidates,
    # --gpu-strip-rows)
    gpuSgm: str = "auto"
    esgmCandidates: int = 2
    gpuStripRows: int = 64
    # pyramid matcher (Options.java:28,85-86; DenseMatcher.java)
    pyramidLevels: int = 1  # 0 = automatic
    pyramidRadius: int = 16
    tileSize: int = 512
    tileOverlap: int = 32
    memoryMb: int = 2048

    def copy(self) -> "Options":
        return copy.copy(self)

    @property
    def window_x(self) -> int:
        return self.census

    @property
    def window_y(self) -> int:
        return self.censusHeight or self.census

    def validate(self) -> "Options":
        """Stereo-path checks of Options.validate (Options.java:766-933)."""
        if self.matchingCost not in ("census", "ad-census", "census-gradient", "zncc"):
            raise ValueError("Unknown matching cost")
        if self.medianMode not in ("edge-preserving", "classic"):
            raise ValueError("--median-mode must be edge-preserving or classic")
        if self.sgmEdgeScale < 0 or self.sgmEdgeScale > 255 or self.medianMaxChange < 0:
            raise ValueError("--sgm-edge-scale must be 0..255; --median-max-change must be nonnegative")
        if (self.medianEdgeThreshold < 0 or self.medianEdgeThreshold > 255
                or self.speckleConnectivity not in (4, 8)):
            raise ValueError("Median edge threshold must be 0..255; speckle connectivity must be 4 or 8")
        if self.sgmAggregate not in ("auto", "16", "32"):
            raise ValueError("--sgm-aggregate must be auto, 16 or 32")
        if not (0 <= self.censusWeight <= 1) or not (1 <= self.adTruncation <= 255) \
                or not (1 <= self.gradientTruncation <= 1020):
            raise ValueError("Invalid matching-cost weight/truncation")
        if (self.correlation < -1 or self.correlation > 1 or self.lrThreshold <= 0
                or self.speckleRange < 0 or self.speckleSize < 0 or self.correlationWindow < 3
                or self.correlationWindow > 15 or self.correlationWindow % 2 == 0):
            raise ValueError("Invalid stereo confidence settings")
        if self.censusMode not in ("gray", "color-distance"):
            raise ValueError("--census-mode must be gray or color-distance")
        if self.p1 != math.floor(self.p1) or self.p2 != math.floor(self.p2):
            raise ValueError("SGM penalties must be integers")
        if (self.disparities < 3 or self.disparities > 4096
                or self.minDisparity + self.disparities > 2**31 - 1):
            raise ValueError("--disparities must be 3..4096 and its upper bound must fit an integer")
        for size in (self.window_x, self.window_y):
            if size < 3 or size > 11 or size % 2 == 0:
                raise ValueError("Census window must be odd, 3..11")
        if self.median < 1 or self.median > 11 or self.median % 2 == 0:
            raise ValueError("Median window must be odd, 1..11")
        if not (0 <= self.p1 < self.p2 <= 1000000) or not (0 <= self.uniqueness < 1):
            raise ValueError("Require 0 <= p1 < p2, 0 <= uniqueness < 1")
        if self.directions not in (4, 8, 16):
            raise ValueError("Directions must be 4 or 8 (16 is this matcher's extension)")
        if self.gpuSgm not in ("auto", "resident", "streamed", "esgm"):
            raise ValueError("--gpu-sgm must be auto, resident, streamed or esgm")
        if self.esgmCandidates < 1 or self.esgmCandidates > 4:
            raise ValueError("--esgm-candidates must be 1..4")
        if self.gpuStripRows < 1:
            raise ValueError("--gpu-strip-rows must be positive")
        if (self.tileSize < 32 or self.tileOverlap < 2 or self.tileOverlap > self.tileSize
                or self.pyramidLevels < 0 or self.pyramidLevels > 6 or self.pyramidRadius < 4
                or self.memoryMb < 16):
            raise ValueError("Invalid tiling / pyramid settings")
        if self.compute not in ("gpu", "auto"):
            raise ValueError("--compute must be gpu or auto for this backend (no CPU fallback)")
        from .stereo_cost import StereoCost

        StereoCost.aggregateBytes(self)
        return self
