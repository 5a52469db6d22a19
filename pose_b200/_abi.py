"""ctypes mirror of include/collinea_sgm.h and the loader of libcollinea_sgm.so.

The library is built in-tree (``pose_b200/libcollinea_sgm.so``).  Loading fails loudly when it is
missing: there is no CPU fallback for the matcher.
"""
from __future__ import annotations

import ctypes
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
LIBRARY_PATH = os.path.join(_HERE, "libcollinea_sgm.so")

CSGM_OK = 0
CSGM_E_INVALID = -1
CSGM_E_CUDA = -2
CSGM_E_NOMEM = -3
CSGM_E_NODEVICE = -4
CSGM_E_TIMEOUT = -5
CSGM_E_BUSY = -6
CSGM_E_UNSUPPORTED = -7

# csgm_session_set_streaming modes (Options.gpuSgm)
CSGM_SGM_AUTO = 0
CSGM_SGM_RESIDENT = 1
CSGM_SGM_STREAMED = 2
CSGM_SGM_COMPACT = 3
SGM_MODES = {"auto": CSGM_SGM_AUTO, "resident": CSGM_SGM_RESIDENT, "streamed": CSGM_SGM_STREAMED,
             "esgm": CSGM_SGM_COMPACT}

STATUS_NAMES = {
    CSGM_E_INVALID: "CSGM_E_INVALID",
    CSGM_E_CUDA: "CSGM_E_CUDA",
    CSGM_E_NOMEM: "CSGM_E_NOMEM",
    CSGM_E_NODEVICE: "CSGM_E_NODEVICE",
    CSGM_E_TIMEOUT: "CSGM_E_TIMEOUT",
    CSGM_E_BUSY: "CSGM_E_BUSY",
    CSGM_E_UNSUPPORTED: "CSGM_E_UNSUPPORTED",
}


class CsgmParams(ctypes.Structure):
    _fields_ = [
        ("disparities", ctypes.c_int32),
        ("min_disparity", ctypes.c_int32),
        ("window_x", ctypes.c_int32),
        ("window_y", ctypes.c_int32),
        ("cost_mode", ctypes.c_int32),
        ("census_weight_milli", ctypes.c_int32),
        ("ad_truncation", ctypes.c_int32),
        ("gradient_truncation", ctypes.c_int32),
        ("p1", ctypes.c_int32),
        ("p2", ctypes.c_int32),
        ("edge_scale", ctypes.c_int32),
        ("directions", ctypes.c_int32),
        ("aggregate_bytes", ctypes.c_int32),
        ("flags", ctypes.c_int32),
        ("uniqueness", ctypes.c_double),
        ("lr_threshold", ctypes.c_double),
    ]


STATS_FIELDS = [
    "lower_boundary_rejected",
    "full_interval_pixels",
    "boundary_rejected",
    "upper_boundary_rejected",
    "ambiguity_rejected",
    "selected",
    "lr_rejected",
    "post_median_lr_rejected",
    "photometric_rejected",
    "speckle_rejected",
    "valid",
]


class CsgmStats(ctypes.Structure):
    _fields_ = [(name, ctypes.c_int64) for name in STATS_FIELDS]


class CsgmPost(ctypes.Structure):
    """csgm_post: the post-filter Options fields (CensusSgm.java:203-272)."""

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


class CsgmDeviceInfo(ctypes.Structure):
    _fields_ = [
        ("name", ctypes.c_char * 256),
        ("memory_bytes", ctypes.c_int64),
        ("sm_count", ctypes.c_int32),
        ("cc_major", ctypes.c_int32),
        ("cc_minor", ctypes.c_int32),
    ]


class CsgmProfile(ctypes.Structure):
    _fields_ = [
        ("kernel_ns", ctypes.c_int64),
        ("upload_ns", ctypes.c_int64),
        ("download_ns", ctypes.c_int64),
        ("uploaded_bytes", ctypes.c_int64),
        ("downloaded_bytes", ctypes.c_int64),
        ("launches", ctypes.c_int64),
        ("calls", ctypes.c_int64),
    ]


class CsgmKernelTime(ctypes.Structure):
    _fields_ = [
        ("name", ctypes.c_char * 32),
        ("launches", ctypes.c_int64),
        ("total_ns", ctypes.c_int64),
    ]


class CsgmTuning(ctypes.Structure):
    _fields_ = [
        ("rows_per_block", ctypes.c_int32),
        ("line_warps", ctypes.c_int32),
        ("line_slack", ctypes.c_int32),
        ("disparity_lanes", ctypes.c_int32),
        ("milliseconds", ctypes.c_double),
    ]


class CsgmError(RuntimeError):
    """A non-zero status from the C ABI, with the library's thread-local message."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


_lib = None
_lock = threading.Lock()

_P = ctypes.c_void_p
_I32 = ctypes.c_int32
_I64 = ctypes.c_int64

# name -> (restype, argtypes); the exported symbols of include/collinea_sgm.h
SIGNATURES = {
    "csgm_version": (ctypes.c_int, []),
    "csgm_last_error": (ctypes.c_char_p, []),
    "csgm_effective_penalties": (
        ctypes.c_int,
        [ctypes.c_double, ctypes.c_double, _I32, _I32, ctypes.POINTER(_I32), ctypes.POINTER(_I32)],
    ),
    "csgm_aggregate_bytes": (
        ctypes.c_int,
        [_I32, _I32, _I32, ctypes.POINTER(_I32), ctypes.POINTER(_I64)],
    ),
    "csgm_device_count": (ctypes.c_int, [ctypes.POINTER(_I32)]),
    "csgm_device_info_get": (ctypes.c_int, [_I32, ctypes.POINTER(CsgmDeviceInfo)]),
    "csgm_session_open": (ctypes.c_int, [_I32, ctypes.POINTER(_P)]),
    "csgm_session_close": (None, [_P]),
    "csgm_session_set_budget": (ctypes.c_int, [_P, _I64]),
    "csgm_session_set_streaming": (ctypes.c_int, [_P, _I32, _I32]),
    "csgm_session_set_candidates": (ctypes.c_int, [_P, _I32]),
    "csgm_session_set_host_budget": (ctypes.c_int, [_P, _I64]),
    "csgm_session_compact_report": (
        ctypes.c_int, [_P, _I32, ctypes.POINTER(_I64), ctypes.POINTER(_I64)]),
    "csgm_plan_detail": (
        ctypes.c_int,
        [_P, ctypes.POINTER(CsgmParams), _I32, _I32, ctypes.POINTER(_I32), ctypes.POINTER(_I64),
         ctypes.POINTER(_I64)],
    ),
    "csgm_plan": (ctypes.c_int, [_P, ctypes.POINTER(CsgmParams), _I32, _I32, ctypes.POINTER(_I64)]),
    "csgm_disparity_limit": (
        ctypes.c_int,
        [_P, ctypes.POINTER(CsgmParams), _I32, _I32, ctypes.POINTER(_I32)],
    ),
    "csgm_profile_get": (ctypes.c_int, [_P, ctypes.POINTER(CsgmProfile), _I32]),
    "csgm_session_set_profiling": (ctypes.c_int, [_P, _I32]),
    "csgm_kernel_times": (
        ctypes.c_int,
        [_P, ctypes.POINTER(CsgmKernelTime), _I32, ctypes.POINTER(_I32), _I32],
    ),
    "csgm_session_synchronize": (ctypes.c_int, [_P]),
    "csgm_autotune": (
        ctypes.c_int,
        [_P, ctypes.POINTER(CsgmParams), _I32, _I32, ctypes.c_char_p, ctypes.POINTER(CsgmTuning)],
    ),
    "csgm_session_load_tuning": (ctypes.c_int, [_P, ctypes.c_char_p]),
    "csgm_session_set_tuning": (ctypes.c_int, [_P, ctypes.POINTER(CsgmTuning)]),
    "csgm_tuning_get": (
        ctypes.c_int,
        [_P, ctypes.POINTER(CsgmParams), _I32, _I32, ctypes.POINTER(CsgmTuning)],
    ),
    "csgm_tuning_cache_lookup": (
        ctypes.c_int,
        [ctypes.c_char_p, ctypes.POINTER(CsgmParams), _I32, _I32, ctypes.POINTER(CsgmTuning)],
    ),
    "csgm_session_set_wait_limit": (ctypes.c_int, [_P, _I64]),
    "csgm_session_set_graphs": (ctypes.c_int, [_P, _I32]),
    "csgm_graph_stats": (ctypes.c_int, [_P, ctypes.POINTER(_I64), ctypes.POINTER(_I64)]),
    "csgm_pair_device": (
        ctypes.c_int,
        [_P, ctypes.POINTER(CsgmParams), _P, _P, _P, _P, _I32, _I32, _P, _P, _P, _P, _P,
         ctypes.POINTER(CsgmStats), _I32],
    ),
    "csgm_match": (
        ctypes.c_int,
        [_P, ctypes.POINTER(CsgmParams), _P, _P, _P, _P, _P, _P, _I32, _I32, _I32, _P, _P, _P, _P,
         ctypes.POINTER(CsgmStats)],
    ),
    "csgm_pair": (
        ctypes.c_int,
        [_P, ctypes.POINTER(CsgmParams), _P, _P, _P, _P, _I32, _I32, _P, _P, _P, _P, _P,
         ctypes.POINTER(CsgmStats)],
    ),
    "csgm_color_census": (ctypes.c_int, [_P, _P, _I32, _I32, _I32, _I32, _P, _P]),
    "csgm_pair_color": (
        ctypes.c_int,
        [_P, ctypes.POINTER(CsgmParams), _P, _P, _P, _P, _P, _P, _I32, _I32, _P, _P, _P, _P, _P,
         ctypes.POINTER(CsgmStats)],
    ),
    "csgm_postfilter_color": (
        ctypes.c_int,
        [_P, ctypes.POINTER(CsgmPost), _P, _P, _P, _P, _P, _I32, _I32, _P, _P,
         ctypes.POINTER(CsgmStats)],
    ),
    "csgm_postfilter": (
        ctypes.c_int,
        [_P, ctypes.POINTER(CsgmPost), _P, _P, _P, _I32, _I32, _P, _P, ctypes.POINTER(CsgmStats)],
    ),
    "csgm_lr_check_noalloc": (
        ctypes.c_int,
        [_P, _P, _I32, _I32, _I32, _I32, ctypes.c_double, _P, _P, _P, _P],
    ),
    "csgm_batch_configure": (ctypes.c_int, [_P, _I32, _I64]),
    "csgm_batch_submit": (
        ctypes.c_int,
        [_P, ctypes.POINTER(CsgmParams), _P, _P, _P, _P, _I32, _I32, _P, _P, _P, _P, _P,
         ctypes.POINTER(_I64)],
    ),
    "csgm_batch_poll": (ctypes.c_int, [_P, _I64, _I32, ctypes.POINTER(CsgmStats)]),
    "csgm_batch_status": (
        ctypes.c_int,
        [_P, ctypes.POINTER(_I32), ctypes.POINTER(_I64), ctypes.POINTER(_I64)],
    ),
    "csgm_host_alloc": (ctypes.c_int, [_I64, ctypes.POINTER(_P)]),
    "csgm_host_free": (None, [_P]),
}


def load() -> ctypes.CDLL:
    """Load libcollinea_sgm.so (once).  Raises if the library has not been built."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIBRARY_PATH):
            raise ImportError(
                f"{LIBRARY_PATH} is missing: build it with `python -m pose_b200.build` "
                "(the matcher has no CPU fallback)"
            )
        lib = ctypes.CDLL(LIBRARY_PATH)
        for name, (restype, argtypes) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = restype
            fn.argtypes = argtypes
        _lib = lib
        return lib


def check(status: int) -> None:
    """Raise CsgmError for a non-zero status."""
    if status != CSGM_OK:
        message = load().csgm_last_error()
        raise CsgmError(status, message.decode() if message else "")
