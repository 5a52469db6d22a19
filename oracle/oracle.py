"""ctypes wrapper of the CPU oracle (liboracle_sgm.so).  TEST INFRASTRUCTURE ONLY.

Only the test suite, ``__graft_entry__.smoke`` and ``bench.py``'s CPU-baseline leg import this
module; the product package never does.  The functions restate the reference's CPU stereo path
(see sgm_oracle.h for the cited lines and for how the restatement is pinned).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

from pose_b200._abi import CsgmParams, CsgmStats

_HERE = os.path.dirname(os.path.abspath(__file__))
LIBRARY_PATH = os.path.join(_HERE, "liboracle_sgm.so")

_P = ctypes.c_void_p
_lib = None


def build() -> str:
    """Compile the oracle with its Makefile (gcc, OpenMP)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return LIBRARY_PATH


def load() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIBRARY_PATH):
            build()
        lib = ctypes.CDLL(LIBRARY_PATH)
        i32, f64 = ctypes.c_int, ctypes.c_double
        lib.oracle_java_round.restype = ctypes.c_int64
        lib.oracle_java_round.argtypes = [f64]
        lib.oracle_words.argtypes = [i32, i32]
        lib.oracle_census.argtypes = [_P, i32, i32, i32, i32, _P]
        lib.oracle_census.restype = None
        lib.oracle_texture.argtypes = [_P, i32, i32, i32, i32, _P]
        lib.oracle_texture.restype = None
        lib.oracle_color_census.argtypes = [_P, i32, i32, i32, i32, _P, _P]
        lib.oracle_color_census.restype = None
        lib.oracle_match.argtypes = [ctypes.POINTER(CsgmParams), _P, _P, _P, _P, _P, _P, i32, i32,
                                     i32, _P, ctypes.POINTER(CsgmStats), _P, _P, _P, _P, _P]
        lib.oracle_lr_check.argtypes = [_P, _P, i32, i32, i32, i32, f64, _P,
                                        ctypes.POINTER(CsgmStats), _P]
        lib.oracle_lr_check.restype = None
        lib.oracle_pair.argtypes = [ctypes.POINTER(CsgmParams), _P, _P, _P, _P, i32, i32, _P, _P,
                                    _P, ctypes.POINTER(CsgmStats), _P, _P]
        lib.oracle_postfilter.argtypes = [_P, _P, _P, _P, i32, i32, _P,
                                          ctypes.POINTER(CsgmStats), _P]
        lib.oracle_postfilter.restype = None
        lib.oracle_pair_color.argtypes = [ctypes.POINTER(CsgmParams), _P, _P, _P, _P, _P, _P, i32,
                                          i32, _P, _P, _P, ctypes.POINTER(CsgmStats), _P, _P]
        lib.oracle_postfilter_color.argtypes = [_P, _P, _P, _P, _P, _P, i32, i32, _P,
                                                ctypes.POINTER(CsgmStats), _P]
        lib.oracle_postfilter_color.restype = None
        lib.oracle_zncc.restype = f64
        lib.oracle_zncc.argtypes = [_P, _P, i32, i32, i32, i32, f64, i32, i32]
        lib.oracle_set_threads.argtypes = [i32]
        lib.oracle_set_threads.restype = None
        _lib = lib
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(_P)


def _u8(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.uint8)


class OraclePost(ctypes.Structure):
    _fields_ = [
        ("median", ctypes.c_int32),
        ("median_classic", ctypes.c_int32),
        ("median_edge_threshold", ctypes.c_int32),
        ("correlation_window", ctypes.c_int32),
        ("speckle_size", ctypes.c_int32),
        ("speckle_connectivity", ctypes.c_int32),
        ("border", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
        ("median_max_change", ctypes.c_double),
        ("correlation", ctypes.c_double),
        ("lr_threshold", ctypes.c_double),
        ("speckle_range", ctypes.c_double),
    ]


def set_threads(n: int) -> None:
    load().oracle_set_threads(int(n))


def java_round(v: float) -> int:
    return int(load().oracle_java_round(float(v)))


def words(wx: int, wy: int) -> int:
    return (wx * wy - 1 + 63) // 64


def census(img, w, h, wx, wy):
    img = _u8(img)
    out = np.zeros(words(wx, wy) * w * h, dtype=np.uint64)
    load().oracle_census(_ptr(img), w, h, wx, wy, _ptr(out))
    return out


def texture(img, w, h, wx, wy):
    img = _u8(img)
    out = np.zeros(w * h, dtype=np.uint8)
    load().oracle_texture(_ptr(img), w, h, wx, wy, _ptr(out))
    return out


def color_census(bgr, w, h, wx, wy):
    bgr = _u8(bgr)
    desc = np.zeros(words(wx, wy) * w * h, dtype=np.uint64)
    tex = np.zeros(w * h, dtype=np.uint8)
    load().oracle_color_census(_ptr(bgr), w, h, wx, wy, _ptr(desc), _ptr(tex))
    return desc, tex


def match(params: CsgmParams, a, b, ga, gb, ta, tb, w, h, reverse, *, want_volumes=False,
          want_summary=False, reasons=None, boundary=None):
    """One view (CensusSgm.match CPU branch).  Returns dict with disp, stats and optional volumes."""
    n, D = w * h, params.disparities
    ga, gb, ta, tb = _u8(ga), _u8(gb), _u8(ta), _u8(tb)
    a = np.ascontiguousarray(a, dtype=np.uint64)
    b = np.ascontiguousarray(b, dtype=np.uint64)
    out = np.empty(n, dtype=np.float32)
    stats = CsgmStats()
    cost = np.empty(n * D, dtype=np.uint16) if want_volumes else None
    agg = np.empty(n * D, dtype=np.uint32) if want_volumes else None
    summary = np.empty(6 * n, dtype=np.int32) if want_summary else None
    rc = load().oracle_match(ctypes.byref(params), _ptr(a), _ptr(b), _ptr(ga), _ptr(gb), _ptr(ta),
                             _ptr(tb), w, h, int(reverse), _ptr(out), ctypes.byref(stats),
                             _ptr(reasons), _ptr(boundary), _ptr(cost), _ptr(agg), _ptr(summary))
    if rc != 0:
        raise ValueError("oracle_match rejected its arguments")
    return {"disp": out, "stats": stats, "cost": cost, "aggregate": agg, "summary": summary}


def lr_check(dl, dr, w, h, rx, ry, threshold, reasons=None):
    out = np.empty(w * h, dtype=np.float32)
    stats = CsgmStats()
    load().oracle_lr_check(_ptr(np.ascontiguousarray(dl, np.float32)),
                           _ptr(np.ascontiguousarray(dr, np.float32)), w, h, rx, ry,
                           float(threshold), _ptr(out), ctypes.byref(stats), _ptr(reasons))
    return out, stats


def pair(params: CsgmParams, left, right, w, h, valid_l=None, valid_r=None, want_reasons=False,
         left_bgr=None, right_bgr=None):
    """Census + both views + LR check (CensusSgm.computeRecorded :56-201); with the BGR images,
    the colour-distance census of --census-mode color-distance."""
    n = w * h
    left, right, valid_l, valid_r = _u8(left), _u8(right), _u8(valid_l), _u8(valid_r)
    checked = np.empty(n, np.float32)
    dl = np.empty(n, np.float32)
    dr = np.empty(n, np.float32)
    reasons = np.empty(n, np.uint8) if want_reasons else None
    boundary = np.empty(n, np.uint8) if want_reasons else None
    stats = CsgmStats()
    if left_bgr is not None:
        lb, rb = _u8(left_bgr), _u8(right_bgr)
        rc = load().oracle_pair_color(ctypes.byref(params), _ptr(left), _ptr(right), _ptr(lb),
                                      _ptr(rb), _ptr(valid_l), _ptr(valid_r), w, h,
                                      _ptr(checked), _ptr(dl), _ptr(dr), ctypes.byref(stats),
                                      _ptr(reasons), _ptr(boundary))
    else:
        rc = load().oracle_pair(ctypes.byref(params), _ptr(left), _ptr(right), _ptr(valid_l),
                                _ptr(valid_r), w, h, _ptr(checked), _ptr(dl), _ptr(dr),
                                ctypes.byref(stats), _ptr(reasons), _ptr(boundary))
    if rc != 0:
        raise ValueError("oracle_pair rejected its arguments")
    return {"checked": checked, "dl": dl, "dr": dr, "stats": stats, "reasons": reasons,
            "boundary": boundary}


def postfilter(post: OraclePost, left, right, dr, w, h, checked, stats: CsgmStats, reasons=None,
               left_bgr=None, right_bgr=None):
    """Median, reciprocity, photometric gate, speckles and the valid count, in place; with the
    BGR images, the three-channel gate of --census-mode color-distance."""
    if left_bgr is not None:
        load().oracle_postfilter_color(ctypes.byref(post), _ptr(_u8(left)), _ptr(_u8(right)),
                                       _ptr(_u8(left_bgr)), _ptr(_u8(right_bgr)),
                                       _ptr(np.ascontiguousarray(dr, np.float32)), w, h,
                                       _ptr(checked), ctypes.byref(stats), _ptr(reasons))
        return
    load().oracle_postfilter(ctypes.byref(post), _ptr(_u8(left)), _ptr(_u8(right)),
                             _ptr(np.ascontiguousarray(dr, np.float32)), w, h, _ptr(checked),
                             ctypes.byref(stats), _ptr(reasons))
