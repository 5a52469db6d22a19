"""The C-ABI library loads and exports every entry point of include/*.h; host-only entry points
behave like the reference's StereoCost helpers; device errors surface as statuses (CPU only)."""
from __future__ import annotations

import ctypes
import glob
import os
import re

import pytest

from pose_b200 import _abi
from pose_b200.options import Options
from pose_b200.stereo_cost import StereoCost

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for header in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(header).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names.update(re.findall(r"^\s*(?:const\s+)?[\w]+[\s\*]+(csgm_\w+)\s*\(", text, flags=re.M))
    return sorted(names)


@pytest.fixture(scope="module")
def lib():
    from pose_b200 import build

    build.build()
    return _abi.load()


def test_every_declared_symbol_is_exported(lib):
    names = declared_functions()
    assert len(names) >= 18, names
    for name in names:
        assert hasattr(lib, name), f"{name} declared in include/ but not exported"
        assert name in _abi.SIGNATURES, f"{name} has no ctypes signature"


def test_version(lib):
    assert lib.csgm_version() == 1


@pytest.mark.parametrize("census,p1,p2,want", [(5, 4, 24, (4, 24)), (11, 4, 24, (20, 120)),
                                               (9, 3, 36, (10, 120)), (7, 4, 24, (8, 48))])
def test_effective_penalties_match_stereo_cost(lib, census, p1, p2, want):
    a, b = ctypes.c_int32(), ctypes.c_int32()
    assert lib.csgm_effective_penalties(p1, p2, census, census, ctypes.byref(a), ctypes.byref(b)) == 0
    o = Options()
    o.census, o.p1, o.p2 = census, p1, p2
    assert (a.value, b.value) == want == (StereoCost.penalty(o.p1, o), StereoCost.p2(o))


def test_aggregate_bytes(lib):
    b, bound = ctypes.c_int32(), ctypes.c_int64()
    assert lib.csgm_aggregate_bytes(8, 24, 0, ctypes.byref(b), ctypes.byref(bound)) == 0
    assert (b.value, bound.value) == (2, 8 * 536)
    assert lib.csgm_aggregate_bytes(8, 24, 32, ctypes.byref(b), ctypes.byref(bound)) == 0
    assert b.value == 4
    assert lib.csgm_aggregate_bytes(16, 7000, 16, ctypes.byref(b), ctypes.byref(bound)) == \
        _abi.CSGM_E_INVALID
    assert b"16-bit" in lib.csgm_last_error()


def test_missing_device_is_a_status(lib):
    """StorageGpuRegression.java:152-165: a missing device index is rejected, not ignored."""
    handle = ctypes.c_void_p()
    assert lib.csgm_session_open(9999, ctypes.byref(handle)) == _abi.CSGM_E_NODEVICE
    assert b"9999" in lib.csgm_last_error()
    from pose_b200.sgm import GpuSgm

    with pytest.raises(_abi.CsgmError) as err:
        GpuSgm(9999)
    assert err.value.status == _abi.CSGM_E_NODEVICE


def test_null_arguments_rejected(lib):
    assert lib.csgm_effective_penalties(4, 24, 5, 5, None, None) == _abi.CSGM_E_INVALID
    assert lib.csgm_device_count(None) == _abi.CSGM_E_INVALID


def test_options_validation():
    o = Options()
    o.directions = 6
    with pytest.raises(ValueError):
        o.validate()
    o = Options()
    o.compute = "cpu"
    with pytest.raises(ValueError, match="no CPU fallback"):
        o.validate()


def test_color_census_rejects_bad_arguments(lib):
    """csgm_color_census validates its arguments on the host before touching a device."""
    assert lib.csgm_color_census(None, None, 64, 64, 5, 5, None, None) == _abi.CSGM_E_INVALID


def test_postfilter_rejects_bad_arguments(lib):
    """csgm_postfilter validates its arguments on the host before touching a device."""
    post = _abi.CsgmPost(median=3, median_classic=0, median_edge_threshold=24,
                         correlation_window=7, speckle_size=50, speckle_connectivity=8, border=4,
                         median_max_change=0.5, correlation=0.55, lr_threshold=0.75,
                         speckle_range=1.0)
    assert lib.csgm_postfilter(None, ctypes.byref(post), None, None, None, 64, 64, None, None,
                               None) == _abi.CSGM_E_INVALID


def test_batch_entry_points_reject_bad_arguments(lib):
    """The batch calls validate their arguments on the host before touching a device."""
    request = ctypes.c_int64()
    assert lib.csgm_batch_configure(None, 4, 0) == _abi.CSGM_E_INVALID
    assert lib.csgm_batch_submit(None, None, None, None, None, None, 64, 64, None, None, None,
                                 None, None, ctypes.byref(request)) == _abi.CSGM_E_INVALID
    assert lib.csgm_batch_poll(None, 1, 0, None) == _abi.CSGM_E_INVALID
    assert lib.csgm_batch_status(None, None, None, None) == _abi.CSGM_E_INVALID
    ptr = ctypes.c_void_p()
    assert lib.csgm_host_alloc(0, ctypes.byref(ptr)) == _abi.CSGM_E_INVALID
