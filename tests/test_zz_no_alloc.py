"""csgm_lr_check_noalloc against the left-right check inside csgm_pair (GPU) and against the
oracle's own views and LR check (CensusSgm.computeRecorded :56-201).

The file name sorts last so the test also runs after every other GPU test has used the device."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from fixtures import upgrade_pair
from pose_b200 import _abi
from pose_b200.options import Options
from pose_b200.stereo_cost import params_from_options

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.asarray(a, np.float32).view(np.uint32)


def test_noalloc_lr_check_matches_pair():
    import torch
    from pose_b200.sgm import GpuSgm

    w, h, _, a, b, ma, mb = upgrade_pair()
    o = Options()
    o.disparities, o.minDisparity = 41, -3
    params = params_from_options(o)
    session = GpuSgm(0)
    try:
        want = session.pair(params, a, b, w, h, ma, mb, want_views=True, want_reasons=True)
    finally:
        session.close()
    lib = _abi.load()
    dev = torch.device("cuda:0")
    dl = torch.from_numpy(want.left.copy()).to(dev)
    dr = torch.from_numpy(want.right.copy()).to(dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    # Two calls in a row: the second one checks that the first left its scratch usable.
    for _ in range(2):
        checked = torch.full((w * h,), 7.0, dtype=torch.float32, device=dev)
        reasons = torch.full((w * h,), 0xEE, dtype=torch.uint8, device=dev)
        count = torch.full((1,), -1, dtype=torch.int64, device=dev)
        _abi.check(lib.csgm_lr_check_noalloc(
            dl.data_ptr(), dr.data_ptr(), w, h, params.window_x, params.window_y,
            params.lr_threshold, checked.data_ptr(), reasons.data_ptr(), count.data_ptr(),
            ctypes.c_void_p(stream)))
        torch.cuda.synchronize(dev)
        # Bit-exact (integer/float selection, no arithmetic tolerance needed).
        assert np.array_equal(_bits(checked.cpu().numpy()), _bits(want.disparity))
        got_reasons = reasons.cpu().numpy()
        assert np.array_equal(got_reasons == 4, want.reasons == 4)
        assert set(np.unique(got_reasons)) <= {4, 0xEE}
        assert int(count.item()) == want.stats.lrRejected


def test_noalloc_lr_check_matches_oracle():
    """The oracle's left and right views through csgm_lr_check_noalloc give the oracle's checked
    map, its reason-4 pixels and its lrRejected count, bit for bit."""
    import torch

    import oracle.oracle as orc

    w, h, _, a, b, ma, mb = upgrade_pair()
    o = Options()
    o.disparities, o.minDisparity = 41, -3
    params = params_from_options(o)
    want = orc.pair(params, a, b, w, h, ma, mb, want_reasons=True)
    lib = _abi.load()
    dev = torch.device("cuda:0")
    dl = torch.from_numpy(want["dl"].copy()).to(dev)
    dr = torch.from_numpy(want["dr"].copy()).to(dev)
    checked = torch.full((w * h,), 7.0, dtype=torch.float32, device=dev)
    reasons = torch.full((w * h,), 0xEE, dtype=torch.uint8, device=dev)
    count = torch.full((1,), -1, dtype=torch.int64, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    _abi.check(lib.csgm_lr_check_noalloc(
        dl.data_ptr(), dr.data_ptr(), w, h, params.window_x, params.window_y,
        params.lr_threshold, checked.data_ptr(), reasons.data_ptr(), count.data_ptr(),
        ctypes.c_void_p(stream)))
    torch.cuda.synchronize(dev)
    assert np.array_equal(_bits(checked.cpu().numpy()), _bits(want["checked"]))
    assert np.array_equal(reasons.cpu().numpy() == 4, want["reasons"] == 4)
    assert int(count.item()) == want["stats"].lr_rejected


def test_noalloc_rejects_heights_beyond_its_scratch():
    import torch

    dev = torch.device("cuda:0")
    w, h = 8, 16385
    buf = torch.zeros(w * h, dtype=torch.float32, device=dev)
    lib = _abi.load()
    status = lib.csgm_lr_check_noalloc(buf.data_ptr(), buf.data_ptr(), w, h, 3, 3, 1.0,
                                       buf.data_ptr(), None, None, None)
    assert status == _abi.CSGM_E_INVALID
    assert b"16384" in lib.csgm_last_error()
