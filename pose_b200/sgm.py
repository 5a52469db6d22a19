"""Host-side mirror of Collinea's matcher interface over the C ABI.

``GpuSgm`` mirrors src/main/java/sgm/GpuSgm.java (device list, session, budget, ``match``,
``disparityLimit``, profiling) and ``CensusSgm`` mirrors src/main/java/sgm/CensusSgm.java
(``compute`` -> ``Result`` with ``Stats``).  Every computation runs in libcollinea_sgm.so on the
GPU; there is no CPU fallback (a missing library or device raises).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import _abi
from ._abi import CsgmDeviceInfo, CsgmParams, CsgmPost, CsgmProfile, CsgmStats, check
from .stereo_cost import params_from_options


def _ptr(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


def _u8(a, n):
    if a is None:
        return None
    a = np.ascontiguousarray(a, dtype=np.uint8).reshape(-1)
    if a.size != n:
        raise ValueError("Invalid stereo image dimensions")
    return a


@dataclass
class Stats:
    """CensusSgm.Stats (CensusSgm.java:683-737)."""

    lowerBoundaryRejected: int = 0
    fullIntervalPixels: int = 0
    boundaryRejected: int = 0
    upperBoundaryRejected: int = 0
    ambiguityRejected: int = 0
    selected: int = 0
    lrRejected: int = 0
    postMedianLrRejected: int = 0
    photometricRejected: int = 0
    speckleRejected: int = 0
    valid: int = 0
    # the pyramid matcher's coarse level (DenseMatcher.java:84-88)
    coarseLowerBoundaryRejected: int = 0
    coarseUpperBoundaryRejected: int = 0
    coarseFullIntervalPixels: int = 0

    _C_NAMES = dict(zip(_abi.STATS_FIELDS, [
        "lowerBoundaryRejected", "fullIntervalPixels", "boundaryRejected",
        "upperBoundaryRejected", "ambiguityRejected", "selected", "lrRejected",
        "postMedianLrRejected", "photometricRejected", "speckleRejected", "valid"]))

    @classmethod
    def from_c(cls, s: CsgmStats) -> "Stats":
        out = cls()
        for c_name, name in cls._C_NAMES.items():
            setattr(out, name, int(getattr(s, c_name)))
        return out

    def to_c(self) -> CsgmStats:
        s = CsgmStats()
        for c_name, name in self._C_NAMES.items():
            setattr(s, c_name, int(getattr(self, name)))
        return s

    def csv(self) -> str:
        """Stats.csv (CensusSgm.java:718-736)."""
        return ",".join(str(v) for v in (
            self.boundaryRejected, self.upperBoundaryRejected, self.ambiguityRejected,
            self.selected, self.lrRejected, self.postMedianLrRejected, self.photometricRejected,
            self.speckleRejected, self.valid))


@dataclass
class Result:
    """CensusSgm.Result (CensusSgm.java:739-767)."""

    width: int
    height: int
    disparity: np.ndarray
    stats: Stats = field(default_factory=Stats)
    left: np.ndarray | None = None
    right: np.ndarray | None = None
    reasons: np.ndarray | None = None
    searchBoundary: np.ndarray | None = None


class GpuSgm:
    """A session on one CUDA device (GpuSgm.java:163-221, closeSession :392-397)."""

    def __init__(self, device: int = 0, memory_mb: int = 0):
        self.lib = _abi.load()
        handle = ctypes.c_void_p()
        check(self.lib.csgm_session_open(int(device), ctypes.byref(handle)))
        self.handle = handle
        self.device = device
        if memory_mb:
            self.set_budget(memory_mb * 1048576)

    # -- lifecycle -------------------------------------------------------------------------
    def close(self) -> None:
        if self.handle:
            self.lib.csgm_session_close(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- devices -----------------------------------------------------------------------------
    @staticmethod
    def devices() -> list:
        """GpuSgm.devices (GpuSgm.java:79-141)."""
        lib = _abi.load()
        count = ctypes.c_int32()
        check(lib.csgm_device_count(ctypes.byref(count)))
        out = []
        for i in range(count.value):
            info = CsgmDeviceInfo()
            check(lib.csgm_device_info_get(i, ctypes.byref(info)))
            out.append({"index": i, "name": info.name.decode(), "memory": info.memory_bytes,
                        "sm_count": info.sm_count, "cc": (info.cc_major, info.cc_minor)})
        return out

    # -- budget and planning -----------------------------------------------------------------
    def set_budget(self, nbytes: int) -> None:
        check(self.lib.csgm_session_set_budget(self.handle, int(nbytes)))

    def set_streaming(self, mode: str = "auto", strip_rows: int = 64) -> None:
        """Options.gpuSgm ("auto", "resident", "streamed", "esgm") and Options.gpuStripRows."""
        check(self.lib.csgm_session_set_streaming(self.handle, _abi.SGM_MODES[mode],
                                                  int(strip_rows)))

    def set_candidates(self, per_path: int = 2) -> None:
        """Options.esgmCandidates: compact SGM's separated proposals per path (1..4)."""
        check(self.lib.csgm_session_set_candidates(self.handle, int(per_path)))

    def set_host_budget(self, nbytes: int) -> None:
        """Host memory for a streamed plan's parked aggregate (0: no limit); over it, auto mode
        runs compact SGM where it applies (GpuCandidateStereo.hostBudget, --memory-mb)."""
        check(self.lib.csgm_session_set_host_budget(self.handle, int(nbytes)))

    def compact_report(self, reverse: int = 0) -> tuple:
        """(certified, verified exactly) pixels of compact SGM's last view of that side."""
        cert, exact = ctypes.c_int64(), ctypes.c_int64()
        check(self.lib.csgm_session_compact_report(self.handle, int(reverse), ctypes.byref(cert),
                                                   ctypes.byref(exact)))
        return cert.value, exact.value

    def plan(self, params: CsgmParams, w: int, h: int) -> int:
        out = ctypes.c_int64()
        check(self.lib.csgm_plan(self.handle, ctypes.byref(params), w, h, ctypes.byref(out)))
        return out.value

    def plan_detail(self, params: CsgmParams, w: int, h: int) -> dict:
        """GpuStereo.plan's Plan (GpuStereo.java:33-84): streamed or resident, strip rows, device
        and pinned host bytes."""
        rows, dev, host = ctypes.c_int32(), ctypes.c_int64(), ctypes.c_int64()
        check(self.lib.csgm_plan_detail(self.handle, ctypes.byref(params), w, h,
                                        ctypes.byref(rows), ctypes.byref(dev),
                                        ctypes.byref(host)))
        return {"streamed": rows.value < h, "rows": rows.value, "device_bytes": dev.value,
                "host_bytes": host.value}

    def disparityLimit(self, params: CsgmParams, w: int, h: int) -> int:
        """GpuSgm.disparityLimit (GpuSgm.java:237-245)."""
        out = ctypes.c_int32()
        check(self.lib.csgm_disparity_limit(self.handle, ctypes.byref(params), w, h,
                                            ctypes.byref(out)))
        return out.value

    # -- profiling ---------------------------------------------------------------------------
    def set_profiling(self, level: int) -> None:
        check(self.lib.csgm_session_set_profiling(self.handle, int(level)))

    def profile(self, reset: bool = False) -> dict:
        """GpuSgm.Compute.profile (GpuSgm.java:592-604)."""
        p = CsgmProfile()
        check(self.lib.csgm_profile_get(self.handle, ctypes.byref(p), int(reset)))
        return {name: getattr(p, name) for name, _ in CsgmProfile._fields_}

    def kernel_times(self, reset: bool = False) -> dict:
        count = ctypes.c_int32()
        records = (_abi.CsgmKernelTime * 64)()
        check(self.lib.csgm_kernel_times(self.handle, records, 64, ctypes.byref(count),
                                         int(reset)))
        return {r.name.decode(): (r.launches, r.total_ns) for r in records[:min(64, count.value)]}

    def synchronize(self) -> None:
        check(self.lib.csgm_session_synchronize(self.handle))

    # -- autotuned launch shapes ----------------------------------------------------------
    @staticmethod
    def _tuning_dict(t) -> dict:
        return {"rows_per_block": t.rows_per_block, "line_warps": t.line_warps,
                "line_slack": t.line_slack, "disparity_lanes": t.disparity_lanes,
                "milliseconds": t.milliseconds}

    def autotune(self, params: CsgmParams, w: int, h: int, cache_path: str | None = None) -> dict:
        """Time the sweep's launch shapes on a synthetic w x h pair and keep the fastest."""
        t = _abi.CsgmTuning()
        path = cache_path.encode() if cache_path else None
        check(self.lib.csgm_autotune(self.handle, ctypes.byref(params), w, h, path,
                                     ctypes.byref(t)))
        return self._tuning_dict(t)

    def load_tuning(self, cache_path: str) -> None:
        check(self.lib.csgm_session_load_tuning(self.handle, cache_path.encode()))

    def set_tuning(self, tuning: dict | None) -> None:
        """Force one launch shape for every call (None: the tuned / default shapes)."""
        if tuning is None:
            check(self.lib.csgm_session_set_tuning(self.handle, None))
            return
        t = _abi.CsgmTuning(tuning.get("rows_per_block", 0), tuning.get("line_warps", -1),
                            tuning.get("line_slack", 0), 0, 0.0)
        check(self.lib.csgm_session_set_tuning(self.handle, ctypes.byref(t)))

    def tuning(self, params: CsgmParams, w: int, h: int) -> dict:
        t = _abi.CsgmTuning()
        check(self.lib.csgm_tuning_get(self.handle, ctypes.byref(params), w, h, ctypes.byref(t)))
        return self._tuning_dict(t)

    def set_graphs(self, enabled: bool) -> None:
        """Capture csgm_pair_device's device pipeline as a CUDA graph and replay it."""
        check(self.lib.csgm_session_set_graphs(self.handle, int(bool(enabled))))

    def graph_stats(self) -> tuple:
        cap, rep = ctypes.c_int64(), ctypes.c_int64()
        check(self.lib.csgm_graph_stats(self.handle, ctypes.byref(cap), ctypes.byref(rep)))
        return cap.value, rep.value

    def set_wait_limit(self, cycles: int) -> None:
        """Watchdog of the device-side waits in SM clock cycles (0 = the default, ~2 s); a wait
        that runs out makes the call fail with CSGM_E_TIMEOUT and leaves the session usable."""
        check(self.lib.csgm_session_set_wait_limit(self.handle, int(cycles)))

    # -- the hot path ------------------------------------------------------------------------
    def match(self, params: CsgmParams, a, b, grayA, grayB, ta, tb, w: int, h: int,
              reverse: bool, stats: Stats | None = None, reasons=None, searchBoundary=None,
              summary: bool = False):
        """GpuSgm.match (GpuSgm.java:267-303): one view from host descriptors and masks.
        Returns the float disparities (and the winners record if ``summary``)."""
        n = w * h
        words = (params.window_x * params.window_y - 1 + 63) // 64
        a = np.ascontiguousarray(a, dtype=np.uint64).reshape(-1)
        b = np.ascontiguousarray(b, dtype=np.uint64).reshape(-1)
        if a.size != words * n or b.size != words * n:
            raise ValueError("descriptor planes do not match the window and image size")
        grayA, grayB, ta, tb = _u8(grayA, n), _u8(grayB, n), _u8(ta, n), _u8(tb, n)
        out = np.empty(n, np.float32)
        rec = np.empty(6 * n, np.int32) if summary else None
        cstats = stats.to_c() if stats is not None else CsgmStats()
        for arr in (reasons, searchBoundary):
            if arr is not None and (arr.dtype != np.uint8 or arr.size != n
                                    or not arr.flags.c_contiguous):
                raise ValueError("reasons/searchBoundary must be contiguous uint8[w*h]")
        check(self.lib.csgm_match(self.handle, ctypes.byref(params), _ptr(a), _ptr(b),
                                  _ptr(grayA), _ptr(grayB), _ptr(ta), _ptr(tb), w, h,
                                  int(bool(reverse)), _ptr(out), _ptr(rec), _ptr(reasons),
                                  _ptr(searchBoundary), ctypes.byref(cstats)))
        if stats is not None:
            for c_name, name in Stats._C_NAMES.items():
                setattr(stats, name, int(getattr(cstats, c_name)))
        return (out, rec) if summary else out

    def pair(self, params: CsgmParams, left, right, w: int, h: int, validLeft=None,
             validRight=None, want_views: bool = False, want_reasons: bool = False,
             leftBgr=None, rightBgr=None) -> Result:
        """Census, both views and the LR check on the GPU (CensusSgm.computeRecorded :56-201);
        with the interleaved BGR images, the colour-distance census (--census-mode
        color-distance, :108-120)."""
        n = w * h
        left, right = _u8(left, n), _u8(right, n)
        validLeft, validRight = _u8(validLeft, n), _u8(validRight, n)
        if (validLeft is None) != (validRight is None):
            raise ValueError("Invalid stereo mask dimensions")
        checked = np.empty(n, np.float32)
        dl = np.empty(n, np.float32) if want_views else None
        dr = np.empty(n, np.float32) if want_views else None
        reasons = np.empty(n, np.uint8) if want_reasons else None
        boundary = np.empty(n, np.uint8) if want_reasons else None
        cstats = CsgmStats()
        if leftBgr is not None or rightBgr is not None:
            if leftBgr is None or rightBgr is None:
                raise ValueError("Color-distance census requires interleaved BGR inputs")
            lb, rb = _u8(leftBgr, 3 * n), _u8(rightBgr, 3 * n)
            check(self.lib.csgm_pair_color(self.handle, ctypes.byref(params), _ptr(left),
                                           _ptr(right), _ptr(lb), _ptr(rb), _ptr(validLeft),
                                           _ptr(validRight), w, h, _ptr(checked), _ptr(dl),
                                           _ptr(dr), _ptr(reasons), _ptr(boundary),
                                           ctypes.byref(cstats)))
        else:
            check(self.lib.csgm_pair(self.handle, ctypes.byref(params), _ptr(left), _ptr(right),
                                     _ptr(validLeft), _ptr(validRight), w, h, _ptr(checked),
                                     _ptr(dl), _ptr(dr), _ptr(reasons), _ptr(boundary),
                                     ctypes.byref(cstats)))
        return Result(w, h, checked, Stats.from_c(cstats), dl, dr, reasons, boundary)

    def color_census(self, bgr, w: int, h: int, window_x: int, window_y: int):
        """CensusSgm.colorCensus (CensusSgm.java:302-332) on the GPU: (descriptors uint64
        [words][w*h], textured uint8 [w*h]) of an interleaved BGR image."""
        n = w * h
        bgr = np.ascontiguousarray(bgr, np.uint8).reshape(-1)
        if bgr.size != 3 * n:
            raise ValueError("bgr must hold 3*w*h bytes")
        words = (window_x * window_y - 1 + 63) // 64
        desc = np.empty((words, n), np.uint64)
        tex = np.empty(n, np.uint8)
        check(self.lib.csgm_color_census(self.handle, _ptr(bgr), w, h, window_x, window_y,
                                         _ptr(desc), _ptr(tex)))
        return desc, tex

    def postfilter(self, post: CsgmPost, left, right, disp_r, w: int, h: int, checked,
                   reasons=None, stats: CsgmStats | None = None, leftBgr=None, rightBgr=None):
        """The post-filters of CensusSgm.computeRecorded (:203-272) on the GPU: median,
        post-median reciprocity, photometric gate, speckles.  `checked` (float32) and `reasons`
        (uint8) are numpy arrays updated in place; `stats` (CsgmStats) is updated like the
        reference's Stats.  With the BGR images the gate correlates their three channels."""
        n = w * h
        left, right = _u8(left, n), _u8(right, n)
        disp_r = np.ascontiguousarray(disp_r, np.float32)
        if checked.dtype != np.float32 or not checked.flags.c_contiguous or checked.size != n:
            raise ValueError("checked must be a contiguous float32 array of w*h values")
        if reasons is not None and (reasons.dtype != np.uint8 or not reasons.flags.c_contiguous
                                    or reasons.size != n):
            raise ValueError("reasons must be a contiguous uint8 array of w*h values")
        if disp_r.size != n:
            raise ValueError("disp_r must hold w*h values")
        st = ctypes.byref(stats) if stats is not None else None
        if leftBgr is not None or rightBgr is not None:
            if leftBgr is None or rightBgr is None:
                raise ValueError("Color-distance census requires interleaved BGR inputs")
            lb, rb = _u8(leftBgr, 3 * n), _u8(rightBgr, 3 * n)
            check(self.lib.csgm_postfilter_color(self.handle, ctypes.byref(post), _ptr(left),
                                                 _ptr(right), _ptr(lb), _ptr(rb), _ptr(disp_r),
                                                 w, h, _ptr(checked), _ptr(reasons), st))
        else:
            check(self.lib.csgm_postfilter(self.handle, ctypes.byref(post), _ptr(left),
                                           _ptr(right), _ptr(disp_r), w, h, _ptr(checked),
                                           _ptr(reasons), st))
        return checked


def post_settings(options) -> CsgmPost:
    """csgm_post from Options: the fields computeRecorded reads after the LR check
    (CensusSgm.java:203-272); the reciprocity radius is census / 2 as there."""
    o = options
    post = CsgmPost()
    post.median = o.median
    post.median_classic = 1 if o.medianMode == "classic" else 0
    post.median_edge_threshold = o.medianEdgeThreshold
    post.correlation_window = o.correlationWindow
    post.speckle_size = o.speckleSize
    post.speckle_connectivity = o.speckleConnectivity
    post.border = o.census // 2
    post.median_max_change = o.medianMaxChange
    post.correlation = o.correlation
    post.lr_threshold = o.lrThreshold
    post.speckle_range = o.speckleRange
    return post


class CensusSgm:
    """CensusSgm (CensusSgm.java:10-280) over a GpuSgm session."""

    def __init__(self, options, session: GpuSgm | None = None):
        self.options = options.validate()
        self._own = session is None
        self.session = session or GpuSgm(options.gpuDevice, options.gpuMemoryMb)
        self.session.set_streaming(options.gpuSgm, options.gpuStripRows)
        self.session.set_candidates(options.esgmCandidates)
        self.session.set_host_budget(options.memoryMb << 20)  # GpuCandidateStereo.hostBudget

    def params(self) -> CsgmParams:
        return params_from_options(self.options)

    def _bgr(self, leftBgr, rightBgr):
        """The BGR images of --census-mode color-distance (CensusSgm.java:108-115)."""
        if self.options.censusMode != "color-distance":
            return None, None
        if leftBgr is None or rightBgr is None:
            raise ValueError("Color-distance census requires interleaved BGR inputs")
        return leftBgr, rightBgr

    def match_pair(self, left, right, width: int, height: int, validLeft=None, validRight=None,
                   want_views=False, want_reasons=False, leftBgr=None, rightBgr=None) -> Result:
        """The matcher up to the LR check (CensusSgm.java:56-201)."""
        o = self.options
        if width < o.window_x + 2 or height < o.window_y + 2:
            raise ValueError("Invalid stereo image dimensions")
        lb, rb = self._bgr(leftBgr, rightBgr)
        return self.session.pair(self.params(), left, right, width, height, validLeft,
                                 validRight, want_views, want_reasons, leftBgr=lb, rightBgr=rb)

    def compute(self, left, right, width: int, height: int, validLeft=None, validRight=None,
                want_reasons=False, leftBgr=None, rightBgr=None) -> Result:
        """CensusSgm.computeRecorded (CensusSgm.java:56-272): the matcher and the LR check, then
        the median, post-median reciprocity, photometric gate and speckle removal, with the
        Stats counters of both stages (colour-distance mode: BGR descriptors and a three-channel
        gate)."""
        lb, rb = self._bgr(leftBgr, rightBgr)
        res = self.match_pair(left, right, width, height, validLeft, validRight,
                              want_views=True, want_reasons=want_reasons, leftBgr=lb,
                              rightBgr=rb)
        cstats = res.stats.to_c()
        self.session.postfilter(post_settings(self.options), left, right, res.right, width,
                                height, res.disparity, res.reasons, cstats, leftBgr=lb,
                                rightBgr=rb)
        res.stats = Stats.from_c(cstats)
        return res

    def close(self):
        if self._own:
            self.session.close()
