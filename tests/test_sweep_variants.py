"""The fused sweep's tuning variants give the same bits as the default.

The sweep reads its tuning knobs once per process (CSGM_SWEEP_ROWS, CSGM_SWEEP_LINE_WARPS,
CSGM_SWEEP_LINE_SLACK), so each variant runs the parity tests of test_gpu_parity.py in a child
process with the knob set: the 1600-pixel cfg1 band against the oracle, and the full-size pair
against the general kernels.  A slack of 10% leaves every anti-diagonal line longer than a tenth
of a block's remaining row to the launch after the sweep, whose warps take them from the queue.
"""
from __future__ import annotations

import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))

VARIANTS = {
    "lines_after_sweep": ({"CSGM_SWEEP_LINE_SLACK": "10"},
                          "test_full_size_cfg1_fused_equals_general or "
                          "(test_pair_band_of_cfg1 and 128)"),
    "four_line_warps": ({"CSGM_SWEEP_LINE_WARPS": "4"},
                        "(test_pair_band_of_cfg1 and 128) or "
                        "(test_full_size_cfg1_fused_equals_general and census-gradient)"),
    "line_kernel": ({"CSGM_SWEEP_LINE_WARPS": "0"}, "test_pair_band_of_cfg1"),
    "eight_rows": ({"CSGM_SWEEP_ROWS": "8"}, "test_pair_band_of_cfg1 and 128"),
}


@pytest.mark.parametrize("name", sorted(VARIANTS))
def test_sweep_variant_matches(name):
    env_extra, selection = VARIANTS[name]
    env = dict(os.environ, **env_extra)
    cmd = [sys.executable, "-m", "pytest", "-q", "-x", "-m", "gpu", "-p", "no:cacheprovider",
           os.path.join(HERE, "test_gpu_parity.py"), "-k", selection]
    run = subprocess.run(cmd, env=env, cwd=os.path.dirname(HERE), capture_output=True, text=True,
                         timeout=600)
    tail = (run.stdout + run.stderr)[-3000:]
    assert run.returncode == 0, f"{name}: child tests failed\n{tail}"
    assert " passed" in run.stdout and " failed" not in run.stdout, tail
