"""B200-native semi-global stereo matcher behind Collinea's matcher interface.

The compute path is libcollinea_sgm.so (hand-written sm_100a CUDA behind a C ABI,
include/collinea_sgm.h).  This package is the host-side mirror of the reference's Java interface
for that path: Options, StereoCost, CensusSgm, and the session that GpuSgm provides.
"""
from .options import Options
from .stereo_cost import StereoCost, params_from_options

__all__ = ["Options", "StereoCost", "params_from_options"]
