"""Byte formats the matcher's callers write: the PFM disparity file of
DenseReconstruction.writeDisparity (DenseReconstruction.java:943-956) and the stereo payload of the
reuse cache (ReuseCache.java:555-621, payload framing :198-203, :235-240).

Both are host-side serialisations of a CensusSgm.Result (pose_b200.sgm.Result); the layouts
follow the reference byte for byte so that files written here and by the reference are
interchangeable.
"""
from __future__ import annotations

import io
import struct

import numpy as np

# ReuseCache payload version word ("SGM2"), ReuseCache.java:201,238.
PAYLOAD_VERSION = 0x53474D32

# The counters of a stereo cache entry, in the order the payload stores them
# (ReuseCache.java:592-607).  The three coarse counters belong to the pyramid matcher, which this
# library does not run: they are written as 0 and ignored on reading.
STAT_NAMES = (
    "lowerBoundaryRejected",
    "fullIntervalPixels",
    "coarseLowerBoundaryRejected",
    "coarseUpperBoundaryRejected",
    "coarseFullIntervalPixels",
    "boundaryRejected",
    "upperBoundaryRejected",
    "ambiguityRejected",
    "selected",
    "lrRejected",
    "postMedianLrRejected",
    "photometricRejected",
    "speckleRejected",
    "valid",
)


def write_disparity_pfm(path, width: int, height: int, disparity) -> None:
    """PFM as DenseReconstruction.writeDisparity writes it: the ASCII header
    "Pf\\n<w> <h>\\n-1.0\\n" (one channel, little-endian scale), then the rows from the bottom
    row up, each as little-endian float32."""
    d = np.ascontiguousarray(disparity, np.float32).reshape(height, width)
    with open(path, "wb") as out:
        out.write(f"Pf\n{width} {height}\n-1.0\n".encode("ascii"))
        out.write(d[::-1].astype("<f4").tobytes())


def read_disparity_pfm(path):
    """(width, height, float32[h*w] in top-down row order) of a one-channel PFM file."""
    with open(path, "rb") as f:
        data = f.read()
    parts = data.split(b"\n", 3)
    if len(parts) < 4 or parts[0] != b"Pf":
        raise ValueError("not a one-channel PFM file")
    width, height = (int(v) for v in parts[1].split())
    scale = float(parts[2])
    dtype = "<f4" if scale < 0 else ">f4"
    rows = np.frombuffer(parts[3], dtype, count=width * height).reshape(height, width)
    return width, height, rows[::-1].astype(np.float32).reshape(-1)


def _floats(out, a) -> None:
    # ReuseCache.floats(DataOutputStream, float[]): length (or -1 for null), then big-endian floats.
    if a is None:
        out.write(struct.pack(">i", -1))
        return
    a = np.ascontiguousarray(a, np.float32).reshape(-1)
    out.write(struct.pack(">i", a.size))
    out.write(a.astype(">f4").tobytes())


def stereo_payload(width: int, height: int, stats, disparity, correlation=None,
                   left_right_error=None) -> bytes:
    """payload.bin of a stereo cache entry (ReuseCache.java:235-240, :575-588): version word,
    width, height, the STAT_NAMES counters as longs, then the disparity, correlation and
    left-right-error rasters; big-endian as java.io.DataOutputStream writes them.  `stats` is a
    pose_b200.sgm.Stats (or any object with the counter attributes; missing ones are 0)."""
    out = io.BytesIO()
    out.write(struct.pack(">iii", PAYLOAD_VERSION, width, height))
    for name in STAT_NAMES:
        out.write(struct.pack(">q", int(getattr(stats, name, 0))))
    _floats(out, disparity)
    _floats(out, correlation)
    _floats(out, left_right_error)
    return out.getvalue()


def read_stereo_payload(data: bytes, width: int, height: int):
    """Parses a stereo payload with the reference's checks (ReuseCache.java:198-203, :557-568,
    :614-621): version word, dimension match, raster lengths, no trailing bytes.  Returns
    (counters dict keyed by STAT_NAMES, disparity, correlation, left_right_error); absent rasters
    are None."""
    view = memoryview(data)
    pos = 0

    def take(fmt):
        nonlocal pos
        size = struct.calcsize(fmt)
        if pos + size > len(view):
            raise ValueError("truncated stereo payload")
        values = struct.unpack_from(fmt, view, pos)
        pos += size
        return values

    (version,) = take(">i")
    if version != PAYLOAD_VERSION:
        raise ValueError("Unknown cache version")
    w, h = take(">ii")
    if w != width or h != height:
        raise ValueError("Stereo cache dimension mismatch")
    counters = {name: take(">q")[0] for name in STAT_NAMES}

    def floats():
        nonlocal pos
        (n,) = take(">i")
        if n == -1:
            return None
        if n != width * height:
            raise ValueError("Invalid raster length")
        if pos + 4 * n > len(view):
            raise ValueError("truncated stereo payload")
        a = np.frombuffer(view, ">f4", count=n, offset=pos).astype(np.float32)
        pos += 4 * n
        return a

    disparity, correlation, lr_error = floats(), floats(), floats()
    if pos != len(view):
        raise ValueError("Trailing cache bytes")
    return counters, disparity, correlation, lr_error
