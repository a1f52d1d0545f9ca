"""B200 wavefront path tracer: host-side mirror of the reference interface.

The renderer itself is libwavefront_b200.so (CUDA, sm_100a) behind the C ABI
of include/wavefront.h; this package marshals scenes and configurations into
that ABI.  See native.py for the entry points and scenes.py for the
synthetic workloads.
"""
from . import abi
from .native import (Batch, DeviceScene, Renderer, Scene, WavefrontError, autotune, camera_struct, check, library,
                     material, render_config)

__all__ = ["abi", "Batch", "DeviceScene", "Renderer", "Scene", "WavefrontError", "autotune", "camera_struct", "check",
           "library", "material", "render_config"]
