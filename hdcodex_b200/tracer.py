"""Python binding of the hdcx C ABI (include/hdcx.h) over libhdcx.so.

``PathTracer`` mirrors the reference's VulkanPathTracer
(include/hdcodex/gpu/vulkan_path_tracer.h:26-52): ``set_scene``,
``set_shading_mode`` / ``get_shading_mode``, ``render`` and ``has_geometry``,
with the same argument meaning. ``render`` returns the cumulative running mean
as a (height, width, 4) float32 array, or None where the reference returns an
empty vector (no geometry or a zero size). A failed call raises
``RuntimeError`` (``ValueError`` for the raster-preview mode), as the
reference throws std::runtime_error / std::invalid_argument.

There is no CPU path: without libhdcx.so or without an sm_100 GPU the
constructor raises.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

from . import _abi
from .scene import Scene

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libhdcx.so")

STATUS = {
    0: "HDCX_OK", 1: "HDCX_ERROR_INVALID_ARGUMENT", 2: "HDCX_ERROR_CUDA", 3: "HDCX_ERROR_OUT_OF_MEMORY",
    4: "HDCX_ERROR_NO_DEVICE", 5: "HDCX_ERROR_UNSUPPORTED", 6: "HDCX_ERROR_TIMEOUT", 7: "HDCX_ERROR_INTERNAL",
}

FUSED, MODULAR, RASTER_PREVIEW = 0, 1, 2

# Every exported entry point of include/hdcx.h: name -> (restype, argtypes).
_P = C.c_void_p
SIGNATURES = {
    "hdcx_abi_version": (C.c_uint32, []),
    "hdcx_abi_struct_sizes": (C.c_uint32, [C.POINTER(C.c_uint64), C.c_uint32]),
    "hdcx_material_defaults": (None, [C.POINTER(_abi.MaterialDesc)]),
    "hdcx_light_defaults": (None, [C.POINTER(_abi.LightDesc)]),
    "hdcx_mesh_defaults": (None, [C.POINTER(_abi.MeshDesc)]),
    "hdcx_probe_devices": (C.c_int, [C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "hdcx_create": (C.c_int, [C.c_int32, C.POINTER(C.c_void_p)]),
    "hdcx_destroy": (None, [_P]),
    "hdcx_last_error": (C.c_char_p, [_P]),
    "hdcx_set_scene": (C.c_int, [_P, _P]),
    "hdcx_set_scene_packed": (C.c_int, [_P, C.POINTER(_abi.PackedScene)]),
    "hdcx_pack_scene": (C.c_int, [_P, C.POINTER(C.c_void_p)]),
    "hdcx_packing_view": (C.POINTER(_abi.PackedScene), [_P]),
    "hdcx_packing_destroy": (None, [_P]),
    "hdcx_has_geometry": (C.c_int32, [_P]),
    "hdcx_set_shading_mode": (C.c_int, [_P, C.c_int32]),
    "hdcx_get_shading_mode": (C.c_int32, [_P]),
    "hdcx_render": (C.c_int, [_P, C.POINTER(_abi.Camera), C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                              C.c_uint32, _P, C.POINTER(C.c_int32)]),
    "hdcx_render_static": (C.c_int, [_P, C.POINTER(_abi.Camera), C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                                     C.c_uint32, _P, C.POINTER(C.c_int32)]),
    "hdcx_render_batch": (C.c_int, [C.POINTER(_abi.BatchJob), C.c_uint32, C.c_uint64]),
    "hdcx_render_batch_ex": (C.c_int, [C.POINTER(_abi.BatchJob), C.c_uint32, C.c_uint64, C.c_uint32]),
    "hdcx_read_rgba": (C.c_int, [_P, C.POINTER(C.c_float), C.c_uint64]),
    "hdcx_get_tuning": (C.c_int, [_P, C.POINTER(_abi.Tuning)]),
    "hdcx_set_tuning": (C.c_int, [_P, C.POINTER(_abi.Tuning)]),
    "hdcx_autotune": (C.c_int, [_P, C.POINTER(_abi.Camera), C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                                C.POINTER(_abi.Tuning)]),
    "hdcx_set_radiance_cache": (C.c_int, [_P, _P, C.c_uint32, C.c_uint32, C.c_uint32]),
    "hdcx_get_radiance_cache_stats": (C.c_int, [_P, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), C.POINTER(C.c_float)]),
    "hdcx_set_radiance_cache_spread": (C.c_int, [_P, C.c_float]),
    "hdcx_nrc_defaults": (None, [C.POINTER(_abi.NrcConfig)]),
    "hdcx_nrc_create": (C.c_int, [C.c_int32, C.POINTER(_abi.NrcConfig), C.POINTER(C.c_void_p)]),
    "hdcx_nrc_destroy": (None, [_P]),
    "hdcx_nrc_last_error": (C.c_char_p, [_P]),
    "hdcx_nrc_grid_parameter_count": (C.c_uint64, [_P]),
    "hdcx_nrc_resolutions": (C.c_int, [_P, C.POINTER(C.c_uint32)]),
    "hdcx_nrc_query": (C.c_int, [_P, _P, C.c_uint32, _P]),
    "hdcx_nrc_train": (C.c_int, [_P, _P, _P, C.c_uint32, C.c_uint32, C.POINTER(C.c_float)]),
    "hdcx_nrc_gradients": (C.c_int, [_P, _P, _P, C.c_uint32, C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "hdcx_nrc_check_wait_timeout": (C.c_int, [_P, C.c_uint32]),
    "hdcx_nrc_get_parameters": (C.c_int, [_P, C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "hdcx_nrc_set_parameters": (C.c_int, [_P, C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "hdcx_read_xyz": (C.c_int, [_P, C.POINTER(C.c_double), C.c_uint64, C.POINTER(C.c_uint64)]),
    "hdcx_device_rgba": (C.c_int, [_P, C.POINTER(C.c_void_p)]),
    "hdcx_trace_primary": (C.c_int, [_P, C.POINTER(_abi.Camera), C.c_uint32, C.c_uint32, C.c_uint32,
                                     C.POINTER(C.c_uint32), C.POINTER(C.c_float)]),
    "hdcx_get_stats": (C.c_int, [_P, C.POINTER(_abi.RenderStats)]),
    "hdcx_set_wave_size": (C.c_int, [_P, C.c_uint64]),
    "hdcx_set_profiling": (C.c_int, [_P, C.c_uint32]),
    "hdcx_set_device_memory_limit": (C.c_int, [C.c_int32, C.c_uint64]),
    "hdcx_get_device_memory_usage": (C.c_int, [C.c_int32, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    "hdcx_test_break_bvh": (C.c_int, [_P]),
    "hdcx_set_texture_lod": (C.c_int, [_P, C.c_uint32]),
    "hdcx_read_texture_level": (C.c_int, [_P, C.c_uint32, C.c_uint32, C.c_void_p, C.c_uint64,
                                          C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
    "hdcx_pack_scene_instanced": (C.c_int, [C.c_void_p, C.POINTER(_abi.InstancerDesc), C.c_uint64,
                                            C.POINTER(C.c_void_p)]),
    "hdcx_set_scene_instanced": (C.c_int, [_P, C.c_void_p, C.POINTER(_abi.InstancerDesc), C.c_uint64]),
    "hdcx_update_instancer_points": (C.c_int, [_P, C.c_uint64, C.POINTER(C.c_float), C.c_uint64]),
    "hdcx_get_scene_info": (C.c_int, [_P, C.POINTER(_abi.SceneInfo)]),
    "hdcx_get_batch_graph_stats": (C.c_int, [C.c_int32, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    "hdcx_render_preview": (C.c_int, [_P, C.POINTER(_abi.Camera), C.c_uint32, C.c_uint32, C.c_void_p,
                                      C.POINTER(C.c_int32)]),
    "hdcx_device_preview": (C.c_int, [_P, C.POINTER(C.c_void_p)]),
    "hdcx_render_async": (C.c_int, [_P, C.POINTER(_abi.Camera), C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                                    C.c_uint32, C.POINTER(C.c_uint64)]),
    "hdcx_wait_render": (C.c_int, [_P, C.c_uint64, C.POINTER(C.c_void_p), C.POINTER(C.c_int32)]),
    "hdcx_set_aovs": (C.c_int, [_P, C.c_uint32]),
    "hdcx_read_aovs": (C.c_int, [_P, C.POINTER(C.c_uint32), C.POINTER(C.c_float), C.c_uint64]),
}

PROFILE_STAGE_TIMES = 1
PROFILE_COUNT_TRAVERSAL = 2

_lib = None


def lib():
    """Loads libhdcx.so (building it first if it is missing and nvcc exists)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            from .build import build
            build()
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def set_device_memory_limit(device: int, limit_bytes: int):
    """hdcx_set_device_memory_limit: the library's device-memory budget on
    `device` (0 removes it)."""
    status = lib().hdcx_set_device_memory_limit(device, limit_bytes)
    if status != 0:
        raise RuntimeError(f"hdcx_set_device_memory_limit failed: {STATUS.get(status, status)}")


def device_memory_usage(device: int):
    """(bytes the library holds on `device`, its budget or 0)."""
    used, limit = C.c_uint64(0), C.c_uint64(0)
    status = lib().hdcx_get_device_memory_usage(device, C.byref(used), C.byref(limit))
    if status != 0:
        raise RuntimeError(f"hdcx_get_device_memory_usage failed: {STATUS.get(status, status)}")
    return int(used.value), int(limit.value)


def batch_graph_stats(device: int = 0):
    """(batch graphs instantiated, batch graphs updated in place) on `device`."""
    inst, upd = C.c_uint64(0), C.c_uint64(0)
    status = lib().hdcx_get_batch_graph_stats(device, C.byref(inst), C.byref(upd))
    if status != 0:
        raise RuntimeError(f"hdcx_get_batch_graph_stats failed: {STATUS.get(status, status)}")
    return int(inst.value), int(upd.value)


def probe_devices():
    """(supported, device_count): HdCodexRendererPlugin::IsSupported's question."""
    sup, cnt = C.c_int32(0), C.c_int32(0)
    lib().hdcx_probe_devices(C.byref(sup), C.byref(cnt))
    return bool(sup.value), int(cnt.value)


class PathTracer:
    """The CUDA path tracer behind the C ABI (see module docstring)."""

    def __init__(self, device: int = 0):
        handle = C.c_void_p()
        status = lib().hdcx_create(device, C.byref(handle))
        if status != 0:
            raise RuntimeError(f"hdcx_create failed: {STATUS.get(status, status)} "
                               "(the hdcx tracer needs an sm_100 GPU; it has no CPU path)")
        self._h = handle
        self.width = 0
        self.height = 0

    def close(self):
        if getattr(self, "_h", None):
            lib().hdcx_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    def _check(self, status: int, what: str):
        if status != 0:
            msg = lib().hdcx_last_error(self._h) or b""
            raise RuntimeError(f"{what} failed: {STATUS.get(status, status)}: {msg.decode()}")

    def set_scene(self, scene: Optional[Scene]):
        if scene is None:
            self._check(lib().hdcx_set_scene(self._h, None), "set_scene")
            return
        holder = scene.to_desc()
        if holder.instancer_count:
            self._check(lib().hdcx_set_scene_instanced(self._h, C.cast(holder.pointer(), C.c_void_p), holder.instancers,
                                                       holder.instancer_count), "set_scene")
        else:
            self._check(lib().hdcx_set_scene(self._h, C.cast(holder.pointer(), C.c_void_p)), "set_scene")

    def update_instancer_points(self, instancer: int, positions):
        """hdcx_update_instancer_points: new object-space points (3 floats each)."""
        p = np.ascontiguousarray(np.asarray(positions, dtype=np.float32).reshape(-1))
        self._check(lib().hdcx_update_instancer_points(self._h, instancer, p.ctypes.data_as(C.POINTER(C.c_float)),
                                                       p.size), "update_instancer_points")

    def set_texture_lod(self, mode: int = 1):
        """hdcx_set_texture_lod: 1 filters material textures at the level ray
        cones give, from mip pyramids built on the GPU; 0 samples level 0."""
        self._check(lib().hdcx_set_texture_lod(self._h, mode), "set_texture_lod")

    def texture_level(self, texture: int, level: int):
        """hdcx_read_texture_level: mip level `level` of a packed texture (h, w, 4) float32."""
        w, h = C.c_uint32(0), C.c_uint32(0)
        self._check(lib().hdcx_read_texture_level(self._h, texture, level, None, 0, C.byref(w), C.byref(h)),
                    "read_texture_level")
        out = np.empty((h.value, w.value, 4), dtype=np.float32)
        self._check(lib().hdcx_read_texture_level(self._h, texture, level, out.ctypes.data_as(C.c_void_p), out.size,
                                                  None, None), "read_texture_level")
        return out

    def scene_info(self) -> dict:
        """hdcx_get_scene_info: triangles, instances, bottom levels, BVH and scene bytes, build times."""
        info = _abi.SceneInfo()
        self._check(lib().hdcx_get_scene_info(self._h, C.byref(info)), "get_scene_info")
        return {name: getattr(info, name) for name, _ in _abi.SceneInfo._fields_}

    def set_shading_mode(self, mode: int):
        if mode == RASTER_PREVIEW:
            raise ValueError("raster preview requires the MaterialX graphics backend")
        self._check(lib().hdcx_set_shading_mode(self._h, mode), "set_shading_mode")

    def get_shading_mode(self) -> int:
        return int(lib().hdcx_get_shading_mode(self._h))

    def has_geometry(self) -> bool:
        return bool(lib().hdcx_has_geometry(self._h))

    def set_profiling(self, flags: int):
        self._check(lib().hdcx_set_profiling(self._h, flags), "set_profiling")

    def set_wave_size(self, paths: int):
        self._check(lib().hdcx_set_wave_size(self._h, paths), "set_wave_size")

    def render(self, camera, width, height, sample_index, max_bounces=8, sample_count=1, out=None):
        """Render(camera, w, h, sampleIndex, maxBounces=8, sampleCount=1)."""
        if out is None:
            out = np.empty((height, width, 4), dtype=np.float32)
        written = C.c_int32(0)
        ptr = out.ctypes.data_as(C.c_void_p) if isinstance(out, np.ndarray) else C.c_void_p(out)
        self._check(lib().hdcx_render(self._h, C.byref(camera), width, height, sample_index, max_bounces,
                                      sample_count, ptr, C.byref(written)), "render")
        if not written.value:
            return None
        self.width, self.height = width, height
        return out

    def render_device(self, camera, width, height, sample_index, max_bounces=8, sample_count=1) -> bool:
        """Renders without a host copy; the image stays in device memory."""
        written = C.c_int32(0)
        self._check(lib().hdcx_render(self._h, C.byref(camera), width, height, sample_index, max_bounces,
                                      sample_count, None, C.byref(written)), "render")
        if written.value:
            self.width, self.height = width, height
        return bool(written.value)

    def render_preview(self, camera, width, height):
        """hdcx_render_preview: the half-resolution two-bounce preview,
        upscaled to width x height on the device; returns the image."""
        out = np.empty((height, width, 4), dtype=np.float32)
        written = C.c_int32(0)
        self._check(lib().hdcx_render_preview(self._h, C.byref(camera), width, height,
                                              out.ctypes.data_as(C.c_void_p), C.byref(written)), "render_preview")
        return out if written.value else None

    def render_async(self, camera, width, height, sample_index, max_bounces=8, sample_count=1) -> int:
        """hdcx_render_async: enqueues a render and its read-back; returns its ticket."""
        ticket = C.c_uint64(0)
        self._check(lib().hdcx_render_async(self._h, C.byref(camera), width, height, sample_index, max_bounces,
                                            sample_count, C.byref(ticket)), "render_async")
        return int(ticket.value)

    def wait_render(self, ticket, width, height):
        """hdcx_wait_render: a copy of the frame's image (None if it wrote nothing)."""
        ptr = C.c_void_p()
        written = C.c_int32(0)
        self._check(lib().hdcx_wait_render(self._h, ticket, C.byref(ptr), C.byref(written)), "wait_render")
        if not written.value:
            return None
        buf = (C.c_float * (width * height * 4)).from_address(ptr.value)
        return np.frombuffer(buf, dtype=np.float32).reshape(height, width, 4).copy()

    def set_aovs(self, flags=3):
        """hdcx_set_aovs: 1 | 2 enables the primary-hit id and depth AOVs, 0 disables them."""
        self._check(lib().hdcx_set_aovs(self._h, flags), "set_aovs")

    def read_aovs(self, width, height):
        """hdcx_read_aovs: (primitive ids uint32 [h, w], depth float32 [h, w])."""
        ids = np.empty((height, width), dtype=np.uint32)
        depth = np.empty((height, width), dtype=np.float32)
        self._check(lib().hdcx_read_aovs(self._h, ids.ctypes.data_as(C.POINTER(C.c_uint32)),
                                         depth.ctypes.data_as(C.POINTER(C.c_float)), width * height), "read_aovs")
        return ids, depth

    def read_xyz(self):
        """(xyz_sum (h, w, 3) float64, samples): FP64 CIE XYZ sums of the accumulation."""
        xyz = np.zeros((self.height, self.width, 3), dtype=np.float64)
        samples = C.c_uint64(0)
        self._check(lib().hdcx_read_xyz(self._h, xyz.ctypes.data_as(C.POINTER(C.c_double)), xyz.size,
                                        C.byref(samples)), "read_xyz")
        return xyz, int(samples.value)

    def trace_primary(self, camera, width, height, sample_number):
        prims = np.zeros((height, width), dtype=np.uint32)
        dist = np.zeros((height, width), dtype=np.float32)
        self._check(lib().hdcx_trace_primary(self._h, C.byref(camera), width, height, sample_number,
                                             prims.ctypes.data_as(C.POINTER(C.c_uint32)),
                                             dist.ctypes.data_as(C.POINTER(C.c_float))), "trace_primary")
        return prims, dist

    def set_radiance_cache(self, cache, prefix_bounces=2, training_paths=1 << 14, train_steps=1):
        """Attach a RadianceCache (None detaches it)."""
        self._check(lib().hdcx_set_radiance_cache(self._h, cache.handle if cache is not None else None, prefix_bounces,
                                                  training_paths, train_steps), "set_radiance_cache")

    def set_radiance_cache_spread(self, factor):
        """hdcx_set_radiance_cache_spread: with factor c > 0, cache-mode paths
        also end at the first vertex where their spread exceeds c times the
        primary footprint (Mueller et al. 2021; the paper uses c = 0.01); the
        prefix stays the latest bounce. 0 ends paths by the prefix alone."""
        self._check(lib().hdcx_set_radiance_cache_spread(self._h, factor), "set_radiance_cache_spread")

    def autotune(self, camera, width, height, max_bounces=8, sample_count=1) -> dict:
        """hdcx_autotune: picks the hit sort, wave size and grid sizes for this
        workload shape (cached per device and shape); returns the tuning."""
        r = _abi.Tuning()
        self._check(lib().hdcx_autotune(self._h, C.byref(camera), width, height, max_bounces, sample_count,
                                        C.byref(r)), "autotune")
        return {name: getattr(r, name) for name, _ in _abi.Tuning._fields_}

    def tuning(self) -> dict:
        r = _abi.Tuning()
        self._check(lib().hdcx_get_tuning(self._h, C.byref(r)), "get_tuning")
        return {name: getattr(r, name) for name, _ in _abi.Tuning._fields_}

    def set_tuning(self, wave_paths=0, trace_blocks_per_sm=16, shade_blocks_per_sm=8, sort_hits=0, sort_rays=0):
        """hdcx_set_tuning: paths per wave (0: automatic), blocks of 128 threads
        per SM for traversal and shading (1-64), sort_hits 1 to shade each
        bounce's hits in material order, sort_rays 1 to trace secondary rays
        in direction order. Images do not depend on these."""
        r = _abi.Tuning(wave_paths=wave_paths, trace_blocks_per_sm=trace_blocks_per_sm,
                        shade_blocks_per_sm=shade_blocks_per_sm, sort_hits=sort_hits, sort_rays=sort_rays)
        self._check(lib().hdcx_set_tuning(self._h, C.byref(r)), "set_tuning")

    def radiance_cache_stats(self) -> dict:
        q, n, loss = C.c_uint64(0), C.c_uint64(0), C.c_float(0.0)
        self._check(lib().hdcx_get_radiance_cache_stats(self._h, C.byref(q), C.byref(n), C.byref(loss)),
                    "get_radiance_cache_stats")
        return {"queries": int(q.value), "samples": int(n.value), "last_loss": float(loss.value)}

    def stats(self) -> dict:
        st = _abi.RenderStats()
        self._check(lib().hdcx_get_stats(self._h, C.byref(st)), "get_stats")
        return {name: getattr(st, name) for name, _ in _abi.RenderStats._fields_}


NRC_QUERY_FLOATS = 12
NRC_WEIGHT_COUNT = 17408
NRC_LEVELS = 16


class RadianceCache:
    """hdcx_nrc: the neural radiance cache (hash grid + tensor-core MLP).
    Query, target and output arguments are device pointers (ints)."""

    def __init__(self, device: int = 0, **config):
        cfg = _abi.NrcConfig()
        lib().hdcx_nrc_defaults(C.byref(cfg))
        for k, v in config.items():
            setattr(cfg, k, v)
        self.config = cfg
        h = C.c_void_p()
        status = lib().hdcx_nrc_create(device, C.byref(cfg), C.byref(h))
        if status != 0:
            raise RuntimeError(f"hdcx_nrc_create failed: {STATUS.get(status, status)}")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().hdcx_nrc_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    def _check(self, status, what):
        if status != 0:
            msg = lib().hdcx_nrc_last_error(self._h) or b""
            raise RuntimeError(f"{what} failed: {STATUS.get(status, status)}: {msg.decode()}")

    @property
    def grid_parameter_count(self) -> int:
        return int(lib().hdcx_nrc_grid_parameter_count(self._h))

    def resolutions(self):
        r = (C.c_uint32 * NRC_LEVELS)()
        self._check(lib().hdcx_nrc_resolutions(self._h, r), "resolutions")
        return list(r)

    def query(self, queries_ptr: int, count: int, out_ptr: int):
        self._check(lib().hdcx_nrc_query(self._h, queries_ptr, count, out_ptr), "query")

    def train(self, queries_ptr: int, targets_ptr: int, count: int, steps: int = 1) -> float:
        loss = C.c_float(0.0)
        self._check(lib().hdcx_nrc_train(self._h, queries_ptr, targets_ptr, count, steps, C.byref(loss)), "train")
        return float(loss.value)

    def gradients(self, queries_ptr: int, targets_ptr: int, count: int):
        mlp = np.zeros(NRC_WEIGHT_COUNT, np.float32)
        grid = np.zeros(self.grid_parameter_count, np.float32)
        self._check(lib().hdcx_nrc_gradients(self._h, queries_ptr, targets_ptr, count,
                                             mlp.ctypes.data_as(C.POINTER(C.c_float)),
                                             grid.ctypes.data_as(C.POINTER(C.c_float))), "gradients")
        return mlp, grid

    def check_wait_timeout(self, polls: int = 1 << 14):
        """Status and message of the deliberately expiring bounded wait."""
        status = lib().hdcx_nrc_check_wait_timeout(self._h, polls)
        return STATUS.get(status, status), (lib().hdcx_nrc_last_error(self._h) or b"").decode()

    def parameters(self):
        mlp = np.zeros(NRC_WEIGHT_COUNT, np.float32)
        grid = np.zeros(self.grid_parameter_count, np.float32)
        self._check(lib().hdcx_nrc_get_parameters(self._h, mlp.ctypes.data_as(C.POINTER(C.c_float)),
                                                  grid.ctypes.data_as(C.POINTER(C.c_float))), "get_parameters")
        return mlp, grid

    def set_parameters(self, mlp, grid):
        mlp = np.ascontiguousarray(mlp, np.float32)
        grid = np.ascontiguousarray(grid, np.float32)
        self._check(lib().hdcx_nrc_set_parameters(self._h, mlp.ctypes.data_as(C.POINTER(C.c_float)),
                                                  grid.ctypes.data_as(C.POINTER(C.c_float))), "set_parameters")


BATCH_CUDA_GRAPH = 1


def render_batch(jobs, path_budget: int = 0, graph: bool = False):
    """hdcx_render_batch over `jobs`: (tracer, camera, width, height,
    sample_index, max_bounces, sample_count, out) tuples, `out` a float32
    (height, width, 4) array, a device pointer (int) or None. Returns the list
    of hdcx_batch_job results (status, written, render_ms per job); raises if
    any job failed."""
    arr = (_abi.BatchJob * len(jobs))()
    keep = []
    for i, (tracer, camera, width, height, sample_index, max_bounces, sample_count, out) in enumerate(jobs):
        b = arr[i]
        b.tracer = tracer.handle
        b.camera = camera
        b.width, b.height = width, height
        b.sample_index, b.max_bounces, b.sample_count = sample_index, max_bounces, sample_count
        if isinstance(out, np.ndarray):
            assert out.dtype == np.float32 and out.size >= width * height * 4 and out.flags.c_contiguous
            keep.append(out)
            b.rgba_out = out.ctypes.data
        else:
            b.rgba_out = out
    status = lib().hdcx_render_batch_ex(arr, len(jobs), path_budget, BATCH_CUDA_GRAPH if graph else 0)
    if status != 0:
        failed = [(i, arr[i].status) for i in range(len(jobs)) if arr[i].status != 0]
        i, st = failed[0]
        msg = lib().hdcx_last_error(jobs[i][0].handle) or b""
        raise RuntimeError(f"render_batch failed: job {i}: {STATUS.get(st, st)}: {msg.decode()}")
    for i, job in enumerate(jobs):
        if arr[i].written:
            job[0].width, job[0].height = job[2], job[3]
    return [{"status": arr[i].status, "written": arr[i].written, "render_ms": arr[i].render_ms}
            for i in range(len(jobs))]


def pack_scene(scene: Scene) -> dict:
    """Host packing of a snapshot (no device needed), as numpy arrays."""
    holder = scene.to_desc()
    handle = C.c_void_p()
    status = lib().hdcx_pack_scene_instanced(C.cast(holder.pointer(), C.c_void_p), holder.instancers,
                                             holder.instancer_count, C.byref(handle))
    if status != 0:
        raise RuntimeError(f"hdcx_pack_scene failed: {STATUS.get(status, status)}")
    try:
        view = lib().hdcx_packing_view(handle).contents
        return _packed_to_dict(view)
    finally:
        lib().hdcx_packing_destroy(handle)


def _packed_to_dict(view: _abi.PackedScene) -> dict:
    def arr(ptr, count, dtype):
        if count == 0 or not ptr:
            return np.zeros(0, dtype=dtype)
        addr = C.cast(ptr, C.c_void_p).value
        raw = (C.c_uint8 * (count * np.dtype(dtype).itemsize)).from_address(addr)
        return np.frombuffer(bytes(raw), dtype=dtype).copy()

    n_lights = max(1, view.light_count)
    out = {
        "vertex_count": view.vertex_count, "triangle_count": view.triangle_count,
        "material_count": view.material_count, "light_count": view.light_count,
        "texture_count": view.texture_count, "opaque": view.opaque,
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
