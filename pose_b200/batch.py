"""Batched and served pairs over a GpuSgm session (csgm_batch_* in include/collinea_sgm.h).

A ``PairBatch`` gives the session N slots.  Each slot holds one pair in flight on its own CUDA
stream with a resident device workspace, so pairs submitted back to back overlap on the GPU.
``submit`` returns None when admission refuses the pair right now (no free slot, or the memory
budget is held by pairs in flight); ``poll`` collects a finished pair.  Inputs and outputs live in
page-locked host buffers owned by the request until it is collected.  Every result is
bit-identical to ``GpuSgm.pair`` on the same inputs.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _abi
from ._abi import CsgmError, CsgmParams, CsgmStats, check
from .sgm import Result, Stats


class PinnedArray:
    """A page-locked host allocation viewed as a numpy array (freed with the object)."""

    def __init__(self, lib, count: int, dtype):
        self._lib = lib
        self.ptr = ctypes.c_void_p()
        nbytes = int(count) * np.dtype(dtype).itemsize
        check(lib.csgm_host_alloc(max(nbytes, 1), ctypes.byref(self.ptr)))
        buf = (ctypes.c_uint8 * max(nbytes, 1)).from_address(self.ptr.value)
        self.array = np.frombuffer(buf, dtype=dtype, count=int(count))

    def __del__(self):
        if getattr(self, "ptr", None) and self.ptr.value:
            self._lib.csgm_host_free(self.ptr)
            self.ptr = ctypes.c_void_p()


@dataclass
class _Request:
    w: int
    h: int
    buffers: dict


class PairBatch:
    """Continuous batching of stereo pairs on one session."""

    def __init__(self, session, slots: int = 4, budget_bytes: int = 0):
        self.session = session
        self.lib = session.lib
        check(self.lib.csgm_batch_configure(session.handle, int(slots), int(budget_bytes)))
        self._requests: dict[int, _Request] = {}

    def submit(self, params: CsgmParams, left, right, w: int, h: int, validLeft=None,
               validRight=None, want_views: bool = False, want_reasons: bool = False):
        """Queue a pair; returns its request id, or None if admission refuses it for now."""
        n = w * h
        if (validLeft is None) != (validRight is None):
            raise ValueError("Invalid stereo mask dimensions")
        b = {"left": PinnedArray(self.lib, n, np.uint8), "right": PinnedArray(self.lib, n, np.uint8),
             "checked": PinnedArray(self.lib, n, np.float32)}
        b["left"].array[:] = np.asarray(left, np.uint8).reshape(-1)
        b["right"].array[:] = np.asarray(right, np.uint8).reshape(-1)
        if validLeft is not None:
            b["vl"] = PinnedArray(self.lib, n, np.uint8)
            b["vr"] = PinnedArray(self.lib, n, np.uint8)
            b["vl"].array[:] = np.asarray(validLeft, np.uint8).reshape(-1)
            b["vr"].array[:] = np.asarray(validRight, np.uint8).reshape(-1)
        if want_views:
            b["dl"] = PinnedArray(self.lib, n, np.float32)
            b["dr"] = PinnedArray(self.lib, n, np.float32)
        if want_reasons:
            b["reasons"] = PinnedArray(self.lib, n, np.uint8)
            b["boundary"] = PinnedArray(self.lib, n, np.uint8)
        return self.submit_pinned(params, b, w, h)

    def submit_pinned(self, params: CsgmParams, buffers: dict, w: int, h: int):
        """Queue a pair whose buffers (``PinnedArray`` values keyed left, right, checked and
        optionally vl, vr, dl, dr, reasons, boundary) are already page-locked."""
        def ptr(key):
            return buffers[key].ptr if key in buffers else None

        request = ctypes.c_int64()
        status = self.lib.csgm_batch_submit(
            self.session.handle, ctypes.byref(params), ptr("left"), ptr("right"), ptr("vl"),
            ptr("vr"), w, h, ptr("checked"), ptr("dl"), ptr("dr"), ptr("reasons"),
            ptr("boundary"), ctypes.byref(request))
        if status == _abi.CSGM_E_BUSY:
            return None
        check(status)
        self._requests[request.value] = _Request(w, h, buffers)
        return request.value

    def poll(self, request: int, wait: bool = True, copy: bool = True) -> Result | None:
        """The finished pair, or None if still running.  With copy=False the result's arrays are
        views of the request's pinned buffers (valid while the caller keeps them)."""
        cstats = CsgmStats()
        status = self.lib.csgm_batch_poll(self.session.handle, int(request), int(bool(wait)),
                                          ctypes.byref(cstats))
        if status == _abi.CSGM_E_BUSY:
            return None
        r = self._requests.pop(request, None)
        check(status)
        b = r.buffers

        def out(key):
            if key not in b:
                return None
            return b[key].array.copy() if copy else b[key].array

        return Result(r.w, r.h, out("checked"), Stats.from_c(cstats), out("dl"), out("dr"),
                      out("reasons"), out("boundary"))

    def status(self) -> dict:
        n, reserved, resident = ctypes.c_int32(), ctypes.c_int64(), ctypes.c_int64()
        check(self.lib.csgm_batch_status(self.session.handle, ctypes.byref(n),
                                         ctypes.byref(reserved), ctypes.byref(resident)))
        return {"in_flight": n.value, "reserved_bytes": reserved.value,
                "resident_bytes": resident.value}

    def in_flight(self) -> list:
        return list(self._requests)


__all__ = ["PairBatch", "PinnedArray", "CsgmError"]
