"""CUDA-graph replay of csgm_pair_device: the first call of a key captures, repeats replay, new
contents of the same device buffers give the new results, a new size captures again, and every
result equals the oracle bit for bit."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

import oracle.oracle as orc
from pose_b200 import _abi
from pose_b200.options import Options
from pose_b200.stereo_cost import params_from_options

pytestmark = pytest.mark.gpu


def run_device(s, prm, left, right, w, h):
    import torch

    dl, dr = torch.from_numpy(left).cuda(), torch.from_numpy(right).cuda()
    out = torch.empty(w * h, dtype=torch.float32, device="cuda")
    stats = _abi.CsgmStats()
    _abi.check(s.lib.csgm_pair_device(s.handle, ctypes.byref(prm), dl.data_ptr(), dr.data_ptr(),
                                      None, None, w, h, out.data_ptr(), None, None, None, None,
                                      ctypes.byref(stats), 1))
    return dl, dr, out, stats


def test_capture_then_replay():
    import torch

    from pose_b200.sgm import GpuSgm
    from pose_b200.synthetic import PairSpec, make_pair

    o = Options()
    o.census, o.censusHeight, o.disparities = 9, 7, 64
    prm = params_from_options(o)
    prm.p1, prm.p2 = 10, 120
    w, h = 320, 160
    pairs = [make_pair(PairSpec(w, h, planes=3, d_min=4, d_max=40, seed=s))[:2] for s in (3, 4)]
    with GpuSgm(0) as s:
        s.set_graphs(True)
        left, right = pairs[0]
        dl, dr, out, _ = run_device(s, prm, left, right, w, h)
        stats = _abi.CsgmStats()

        def again(l_img, r_img):
            dl.copy_(torch.from_numpy(l_img))
            dr.copy_(torch.from_numpy(r_img))
            _abi.check(s.lib.csgm_pair_device(s.handle, ctypes.byref(prm), dl.data_ptr(),
                                              dr.data_ptr(), None, None, w, h, out.data_ptr(),
                                              None, None, None, None, ctypes.byref(stats), 1))
            return out.cpu().numpy()

        assert s.graph_stats() == (1, 0)
        for i in range(4):
            l_img, r_img = pairs[i % 2]
            got = again(l_img, r_img)
            want = orc.pair(prm, l_img, r_img, w, h)
            assert np.array_equal(got.view(np.uint32), want["checked"].view(np.uint32)), i
            assert stats.selected == want["stats"].selected
        assert s.graph_stats() == (1, 4)
        # A new size is a new key: plain run plus capture, then replay.
        big = make_pair(PairSpec(400, 200, planes=3, d_min=4, d_max=40, seed=5))[:2]
        for _ in range(2):
            _, _, out2, _ = run_device(s, prm, big[0], big[1], 400, 200)
            want = orc.pair(prm, big[0], big[1], 400, 200)
            assert np.array_equal(out2.cpu().numpy().view(np.uint32),
                                  want["checked"].view(np.uint32))
        captured, replayed = s.graph_stats()
        assert captured >= 2
        s.set_graphs(False)
