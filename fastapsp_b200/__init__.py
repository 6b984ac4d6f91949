"""fastapsp_b200 -- B200-native (sm_100a) per-subgraph APSP solve path of
Fast APSP, behind the reference's fap::fapGraph API.

The compute path is the in-tree shared library libfap_b200.so (CUDA kernels
for stages 1-3 behind a C ABI).  This package is its Python mirror:

    from fastapsp_b200 import fapGraph
"""
from ._lib import (FAP_DTYPE_AUTO, FAP_DTYPE_F32, FAP_DTYPE_I32, FAP_INF_F32, FAP_INF_I32,
                   FAP_MODE_BATCHED, FAP_MODE_PLAIN, FapError)
from .graph import Context, DeviceGraph, fapGraph

__all__ = ["fapGraph", "Context", "DeviceGraph", "FapError", "FAP_DTYPE_AUTO", "FAP_DTYPE_I32",
           "FAP_DTYPE_F32", "FAP_MODE_PLAIN", "FAP_MODE_BATCHED", "FAP_INF_I32", "FAP_INF_F32"]
