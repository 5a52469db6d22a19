"""java.util.Random restated from its published specification (the 48-bit LCG of the Javadoc).

The reference's stereo regressions build their fixtures with ``new Random(seed).nextBytes(buf)``
(e.g. src/test/java/sgm/SelfTest.java:82-86); this class regenerates those bytes exactly so the
fixtures need no JDK.
"""
from __future__ import annotations

import numpy as np

_MULT = 0x5DEECE66D
_ADD = 0xB
_MASK = (1 << 48) - 1


class JavaRandom:
    def __init__(self, seed: int):
        self.seed = (seed ^ _MULT) & _MASK

    def next(self, bits: int) -> int:
        self.seed = (self.seed * _MULT + _ADD) & _MASK
        r = self.seed >> (48 - bits)
        if r & (1 << (bits - 1)) and bits == 32:
            r -= 1 << 32
        return r

    def nextInt(self) -> int:
        return self.next(32)

    def nextBytes(self, n: int) -> np.ndarray:
        """Random.nextBytes: each nextInt() yields up to four bytes, low byte first."""
        out = np.empty(n, dtype=np.uint8)
        i = 0
        while i < n:
            rnd = self.nextInt() & 0xFFFFFFFF
            for _ in range(min(n - i, 4)):
                out[i] = rnd & 0xFF
                rnd >>= 8
                i += 1
        return out
