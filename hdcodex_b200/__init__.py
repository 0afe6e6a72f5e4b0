"""hdcodex_b200 - B200-native (sm_100a) spectral path-tracing backend for hdCodex.

The product is libhdcx.so (C ABI in include/hdcx.h; C++ drop-in
hdcodex::CudaPathTracer in include/hdcx/cuda_path_tracer.h). This package holds
its CUDA sources (csrc/), the build script and a Python binding used by the
tests and the benchmark: ``PathTracer`` mirrors the reference's
VulkanPathTracer and ``scene`` mirrors its SceneSnapshot types.
"""
from . import scene
from .scene import (AUTOMATIC, CYLINDER, DISK, DISTANT, DOME, LATLONG, RECT, SPHERE, Instancer, Light, Material,
                    Mesh, Scene, Texture, camera)
from .tracer import FUSED, MODULAR, RASTER_PREVIEW, PathTracer, lib, pack_scene, probe_devices, render_batch, RadianceCache

__all__ = [
    "scene", "Scene", "Mesh", "Material", "Texture", "Light", "Instancer", "camera", "PathTracer", "pack_scene",
    "render_batch", "RadianceCache",
    "probe_devices", "lib", "FUSED", "MODULAR", "RASTER_PREVIEW", "DOME", "RECT", "DISK", "SPHERE",
    "CYLINDER", "DISTANT", "AUTOMATIC", "LATLONG",
]
