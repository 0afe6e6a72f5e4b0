"""ctypes binding of the CPU oracle (oracle/_build/libhdcx_oracle.so).

TEST INFRASTRUCTURE ONLY. The oracle is a CPU restatement of hdCodex's GLSL
integrator (src/gpu/vulkan_path_tracer.cpp:100-1891) and scene packing; the
tests, ``__graft_entry__.smoke()`` and the benchmark's CPU-baseline leg use it
as the checker. The product (``hdcodex_b200``) never imports it.

``OracleTracer`` has the methods of the reference's VulkanPathTracer
(vulkan_path_tracer.h:26-52): set_scene, has_geometry and render, which returns
the cumulative RGBA32F running mean as a (height, width, 4) array, or None when
the reference would return an empty vector.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from hdcodex_b200 import _abi
from hdcodex_b200.scene import Scene

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libhdcx_oracle.so")


def build(force: bool = False) -> str:
    """Compiles the oracle with its Makefile (g++, -ffp-contract=off)."""
    if force or not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    else:
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        L.oracle_create.restype = C.c_void_p
        L.oracle_destroy.argtypes = [C.c_void_p]
        L.oracle_set_scene.argtypes = [C.c_void_p, C.c_void_p]
        L.oracle_has_geometry.argtypes = [C.c_void_p]
        L.oracle_packed_view.argtypes = [C.c_void_p, C.POINTER(_abi.PackedScene)]
        L.oracle_render.argtypes = [
            C.c_void_p, C.POINTER(_abi.Camera), C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
            C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_int32,
            C.POINTER(C.c_float), C.POINTER(C.c_double), C.POINTER(C.c_uint64)]
        L.oracle_trace_primary.argtypes = [
            C.c_void_p, C.POINTER(_abi.Camera), C.c_uint32, C.c_uint32, C.c_uint32, C.c_int32,
            C.POINTER(C.c_uint32), C.POINTER(C.c_float)]
        _lib = L
    return _lib


class OracleTracer:
    def __init__(self):
        self._h = lib().oracle_create()
        self.width = 0
        self.height = 0
        self.last_counters = (0, 0, 0)

    def __del__(self):
        if getattr(self, "_h", None):
            lib().oracle_destroy(self._h)
            self._h = None

    def set_scene(self, scene: Scene | None):
        if scene is None:
            lib().oracle_set_scene(self._h, None)
            return
        if scene.instancers:  # the oracle renders the flattened scene (hdcx_instancer_desc)
            scene = scene.flattened()
        holder = scene.to_desc()
        lib().oracle_set_scene(self._h, C.cast(holder.pointer(), C.c_void_p))

    def has_geometry(self) -> bool:
        return bool(lib().oracle_has_geometry(self._h))

    def render(self, camera, width, height, sample_index, max_bounces=8, sample_count=1,
               crop=None, threads=0, want_xyz=False):
        rgba = np.zeros((height, width, 4), dtype=np.float32)
        xyz = np.zeros((height, width, 3), dtype=np.float64)
        counters = (C.c_uint64 * 3)()
        x0, y0, x1, y1 = crop if crop else (0, 0, 0, 0)
        ok = lib().oracle_render(
            self._h, C.byref(camera), width, height, sample_index, max_bounces, sample_count,
            x0, y0, x1, y1, threads,
            rgba.ctypes.data_as(C.POINTER(C.c_float)), xyz.ctypes.data_as(C.POINTER(C.c_double)),
            counters)
        self.last_counters = tuple(int(c) for c in counters)
        if not ok:
            return (None, None) if want_xyz else None
        return (rgba, xyz) if want_xyz else rgba

    def trace_primary(self, camera, width, height, sample_number, threads=0):
        prims = np.zeros((height, width), dtype=np.uint32)
        dist = np.zeros((height, width), dtype=np.float32)
        ok = lib().oracle_trace_primary(
            self._h, C.byref(camera), width, height, sample_number, threads,
            prims.ctypes.data_as(C.POINTER(C.c_uint32)), dist.ctypes.data_as(C.POINTER(C.c_float)))
        if not ok:
            return None, None
        return prims, dist

    def packed(self) -> dict:
        """Copies of the packed scene buffers, keyed like hdcx_packed_scene."""
        view = _abi.PackedScene()
        lib().oracle_packed_view(self._h, C.byref(view))
        return packed_view_to_dict(view)


def packed_view_to_dict(view: _abi.PackedScene) -> dict:
    def arr(ptr, count, dtype):
        if count == 0 or not ptr:
            return np.zeros(0, dtype=dtype)
        addr = C.cast(ptr, C.c_void_p).value
        buf = (C.c_uint8 * (count * np.dtype(dtype).itemsize)).from_address(addr)
        return np.frombuffer(bytes(buf), dtype=dtype).copy()

    n_lights = max(1, view.light_count)
    out = {
        "vertex_count": view.vertex_count,
        "triangle_count": view.triangle_count,
        "material_count": view.material_count,
        "light_count": view.light_count,
        "texture_count": view.texture_count,
        "opaque": view.opaque,
        "vertices": arr(view.vertices, view.vertex_count * 4, np.float32),
        "indices": arr(view.indices, view.triangle_count * 3, np.uint32),
        "triangle_materials": arr(view.triangle_materials, view.triangle_count, np.uint32),
        "texcoords": arr(view.texcoords, view.triangle_count * 6, np.float32),
        "normals": arr(view.normals, view.triangle_count * 12, np.float32),
        "materials": arr(view.materials, view.material_count * _abi.GPU_MATERIAL_BYTES, np.uint8),
        "lights": arr(view.lights, n_lights * _abi.GPU_LIGHT_BYTES, np.uint8),
        "emissive": arr(view.emissive, view.triangle_count * 4, np.float32),
        "textures": [],
    }
    for i in range(view.texture_count):
        t = view.textures[i]
        n = t.width * t.height * 4
        dtype = np.float32 if t.format == 2 else np.uint8
        out["textures"].append((t.width, t.height, t.format, arr(t.texels, n, dtype)))
    return out


# ---------------------------------------------------------------------------
# The reference integrator's own GLSL, compiled as C++ by oracle/ref_build.py
# into oracle/_ref/libhdcx_ref.so (built only where the reference checkout is
# present; the library then travels with the repository snapshot).
# ---------------------------------------------------------------------------
REF_LIB_PATH = os.path.join(HERE, "_ref", "libhdcx_ref.so")
_ref_lib = None


def ref_available() -> bool:
    return os.path.exists(REF_LIB_PATH)


def ref_lib():
    global _ref_lib
    if _ref_lib is None:
        L = C.CDLL(REF_LIB_PATH)
        L.ref_create.restype = C.c_void_p
        L.ref_destroy.argtypes = [C.c_void_p]
        L.ref_set_scene.argtypes = [C.c_void_p, C.c_void_p]
        L.ref_render.argtypes = [
            C.c_void_p, C.POINTER(_abi.Camera), C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
            C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_int32, C.POINTER(C.c_float)]
        _ref_lib = L
    return _ref_lib


class ReferenceTracer:
    """VulkanPathTracer's shader run on the CPU (same methods as OracleTracer)."""

    def __init__(self):
        self._h = ref_lib().ref_create()

    def __del__(self):
        if getattr(self, "_h", None):
            ref_lib().ref_destroy(self._h)
            self._h = None

    def set_scene(self, scene: Scene | None):
        if scene is None:
            ref_lib().ref_set_scene(self._h, None)
            return
        if scene.instancers:  # the reference's Hydra adapter flattens instancers
            scene = scene.flattened()
        holder = scene.to_desc()
        ref_lib().ref_set_scene(self._h, C.cast(holder.pointer(), C.c_void_p))

    def render(self, camera, width, height, sample_index, max_bounces=8, sample_count=1, crop=None, threads=0):
        rgba = np.zeros((height, width, 4), dtype=np.float32)
        x0, y0, x1, y1 = crop if crop else (0, 0, 0, 0)
        ok = ref_lib().ref_render(self._h, C.byref(camera), width, height, sample_index, max_bounces,
                                  sample_count, x0, y0, x1, y1, threads,
                                  rgba.ctypes.data_as(C.POINTER(C.c_float)))
        return rgba if ok else None
