"""phosphor_b200 — B200-native (sm_100a) SPPM renderer core behind a C ABI (include/phx.h).

The compute path is libphx.so (hand-written CUDA kernels); this package only loads it and exposes
the reference renderer's host API (ArgsList / Renderer / SceneData) on top of the C ABI.
"""
from . import _capi as capi
from ._capi import PhxError, load
from .renderer import (ArgsList, Batch, Renderer, SceneData, TraversalBvh, bvh_build, camera_make, traversal_bvh,
                       write_png)

__all__ = ["capi", "load", "PhxError", "ArgsList", "Renderer", "Batch", "SceneData", "TraversalBvh", "bvh_build",
           "camera_make", "traversal_bvh", "write_png"]
