"""Failure detection with faults injected on the host: every case returns a
status (the C++ shim's std::runtime_error) and leaves the tracer usable; no
case faults, traps or hangs the GPU.

* a device-memory budget too small for the scene (hdcx_set_device_memory_limit):
  HDCX_ERROR_OUT_OF_MEMORY from set_scene and from a render whose buffers do
  not fit, then normal renders once the budget is lifted;
* a packed scene with an out-of-range vertex or material index
  (hdcx_set_scene_packed): HDCX_ERROR_INVALID_ARGUMENT;
* a snapshot mesh with an out-of-range index: the mesh is dropped by the
  packing, as by the oracle's restatement of BuildScene, and both report no
  geometry;
* NaN vertex coordinates: such triangles are never hit (every comparison of
  the watertight test is false); the render equals the oracle's;
* a cyclic BVH (hdcx_test_break_bvh, every access in bounds): traversal runs
  out of its node budget or stack, the render returns HDCX_ERROR_INTERNAL
  with "traversal fault", and a new set_scene renders normally.
"""
import ctypes as C

import numpy as np
import pytest

import ref_scenes as R
from hdcodex_b200 import PathTracer, workloads
from hdcodex_b200.tracer import device_memory_usage, lib, set_device_memory_limit

pytestmark = pytest.mark.gpu


def test_memory_budget_fails_cleanly_then_recovers():
    wl = workloads.closed_box(width=64, height=64)
    with PathTracer(0) as t:
        used, _ = device_memory_usage(0)
        set_device_memory_limit(0, used + 4096)
        try:
            with pytest.raises(RuntimeError, match="OUT_OF_MEMORY"):
                t.set_scene(wl.scene)
            assert not t.has_geometry()
        finally:
            set_device_memory_limit(0, 0)
        t.set_scene(wl.scene)
        # Room for the scene but not for the render's image and path buffers.
        used, _ = device_memory_usage(0)
        set_device_memory_limit(0, used + 4096)
        try:
            with pytest.raises(RuntimeError, match="OUT_OF_MEMORY"):
                t.render(wl.camera, 64, 64, 0, 8, 2)
        finally:
            set_device_memory_limit(0, 0)
        img = t.render(wl.camera, 64, 64, 0, 8, 2)
        assert np.isfinite(img).all() and float(img[..., :3].mean()) > 0.0
        used, limit = device_memory_usage(0)
        assert used > 0 and limit == 0


@pytest.mark.parametrize("field", ["indices", "triangle_materials"])
def test_packed_scene_with_out_of_range_index_is_rejected(field):
    holder = R.base_scene().to_desc()
    handle = C.c_void_p()
    assert lib().hdcx_pack_scene(C.cast(holder.pointer(), C.c_void_p), C.byref(handle)) == 0
    try:
        view = lib().hdcx_packing_view(handle).contents
        count = view.vertex_count if field == "indices" else view.material_count
        getattr(view, field)[0] = count + 7  # the library's own host copy of the packing
        with PathTracer(0) as t:
            with pytest.raises(RuntimeError, match="INVALID_ARGUMENT.*out of range"):
                t._check(lib().hdcx_set_scene_packed(t.handle, C.byref(view)), "set_scene_packed")
            assert not t.has_geometry()
            t.set_scene(R.base_scene())
            assert t.render(R.base_camera(), 16, 16, 0, 8, 1) is not None
    finally:
        lib().hdcx_packing_destroy(handle)


def test_snapshot_mesh_with_out_of_range_index_is_dropped(oracle_lib):
    scene = R.base_scene()
    idx = list(scene.meshes[0].indices)
    idx[0] = 999
    scene.meshes[0].indices = idx
    o = oracle_lib.OracleTracer()
    o.set_scene(scene)
    with PathTracer(0) as t:
        t.set_scene(scene)
        assert not t.has_geometry() and not o.has_geometry()
        assert t.render(R.base_camera(), 16, 16, 0, 8, 1) is None


def test_nan_vertices_are_never_hit(oracle_lib):
    wl = workloads.closed_box(width=48, height=48)
    pos = list(wl.scene.meshes[-1].positions)
    pos[0] = float("nan")
    pos[4] = float("nan")
    wl.scene.meshes[-1].positions = pos
    o = oracle_lib.OracleTracer()
    o.set_scene(wl.scene)
    ref = o.render(wl.camera, 48, 48, 0, 8, 2)
    with PathTracer(0) as t:
        t.set_scene(wl.scene)
        img = t.render(wl.camera, 48, 48, 0, 8, 2)
    assert np.isfinite(img).all()
    same = float(np.all(img == ref, axis=-1).mean())
    assert same >= 0.99, same


def test_cyclic_bvh_is_reported_not_hung():
    wl = workloads.spectral_stress(width=64, height=36, spp=1, dome_size=(64, 32))
    with PathTracer(0) as t:
        t.set_scene(wl.scene)
        good = t.render(wl.camera, wl.width, wl.height, 0, 8, 1).copy()
        assert lib().hdcx_test_break_bvh(t.handle) == 0
        with pytest.raises(RuntimeError, match="INTERNAL.*traversal fault"):
            t.render(wl.camera, wl.width, wl.height, 0, 8, 1)
        t.set_scene(wl.scene)
        again = t.render(wl.camera, wl.width, wl.height, 0, 8, 1)
        assert np.array_equal(good, again)


def test_break_bvh_needs_eight_nodes():
    with PathTracer(0) as t:
        t.set_scene(R.base_scene())  # one triangle: a single node
        assert lib().hdcx_test_break_bvh(t.handle) == 1
