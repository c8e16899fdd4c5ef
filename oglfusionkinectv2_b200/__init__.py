"""B200-native KinectFusion core with the gFusion / MCubes surface of
philipNoonan/oglFusionKinectV2 (C ABI in include/kf.h, CUDA kernels in csrc/)."""
from . import _lib
from ._lib import KfError, load
from .gfusion import GFusion, GFusionBatch, GFusionConfig, GFusionServer, Intrinsics, MCubes, decode_volume, prefix_sum_device

__all__ = ["GFusion", "GFusionBatch", "GFusionConfig", "GFusionServer", "Intrinsics", "MCubes", "KfError", "load",
           "decode_volume", "prefix_sum_device", "_lib"]
