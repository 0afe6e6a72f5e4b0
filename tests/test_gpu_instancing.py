"""Instancers on the GPU: a scene given with instancers renders exactly as its
flattened snapshot (the oracle's input), through the two-level BVH.

* primary hit triangles and distances bit-exact against the oracle on the
  flattened scene (ids in the flattened numbering), images at the parity
  tolerance; stochastic opacity and the any-hit shadow rules included;
* the 1.0M-triangle heavy scene with its spheres as 256 instances of four
  prototypes: primary ids bit-exact, a render at the parity tolerance, and a
  smaller BVH than the flattened scene's;
* a deforming instanced mesh (hdcx_update_instancer_points: flattened
  vertices recomputed, BLAS refitted, top level rebuilt) renders as the
  flattened scene with the moved points.
"""
import numpy as np
import pytest

import ref_scenes as R
from hdcodex_b200 import Instancer, PathTracer, workloads
from test_instancing import instanced_scene

pytestmark = pytest.mark.gpu

MIN_IDENTICAL = 0.99
MAX_REL_L1 = 1e-3


def close(img, ref):
    same = float(np.all(img == ref, axis=-1).mean())
    rel = float(np.abs(img[..., :3] - ref[..., :3]).sum()) / (float(np.abs(ref[..., :3]).sum()) + 1e-12)
    return same >= MIN_IDENTICAL and rel <= MAX_REL_L1, (same, rel)


def box_with_instances(seed, opacity=1.0):
    """The closed box with the proto sphere instanced inside it."""
    rng = np.random.default_rng(seed)
    wl = workloads.closed_box(width=64, height=64)
    proto = instanced_scene(seed).meshes[0]
    wl.scene.meshes.append(proto)
    Ts = []
    for _ in range(12):
        A = np.eye(3) * rng.uniform(0.05, 0.12) + rng.normal(scale=0.02, size=(3, 3))
        M = np.zeros((4, 4))
        M[:3, :3] = A
        M[3, :3] = rng.uniform(0.2, 0.8, 3)
        M[3, 3] = 1.0
        Ts.append(M)
    wl.scene.instancers = [Instancer(proto.id, np.array(Ts))]
    if opacity < 1.0:
        wl.scene.materials[0].opacity = opacity
    return wl


@pytest.mark.parametrize("seed", range(4))
def test_instanced_box_equals_flattened(oracle_lib, seed):
    wl = box_with_instances(seed)
    o = oracle_lib.OracleTracer()
    o.set_scene(wl.scene)  # the oracle flattens
    ref = o.render(wl.camera, 64, 64, 0, 8, 4)
    rp, rd = o.trace_primary(wl.camera, 64, 64, 1)
    with PathTracer(0) as t:
        t.set_scene(wl.scene)
        info = t.scene_info()
        assert info["instances"] == 13 and info["bottom_levels"] == 2
        p, d = t.trace_primary(wl.camera, 64, 64, 1)
        assert np.array_equal(p, rp) and np.array_equal(d.view(np.uint32), rd.view(np.uint32))
        assert (rp >= 34).sum() > 50  # instanced triangles are seen
        img = t.render(wl.camera, 64, 64, 0, 8, 4)
    ok, info = close(img, ref)
    assert ok, info


def test_instanced_partial_opacity_equals_flattened(oracle_lib):
    wl = box_with_instances(7, opacity=0.6)
    o = oracle_lib.OracleTracer()
    o.set_scene(wl.scene)
    ref = o.render(wl.camera, 64, 64, 0, 8, 4)
    with PathTracer(0) as t:
        t.set_scene(wl.scene)
        img = t.render(wl.camera, 64, 64, 0, 8, 4)
        p, d = t.trace_primary(wl.camera, 64, 64, 0)
    rp, rd = o.trace_primary(wl.camera, 64, 64, 0)
    assert np.array_equal(p, rp) and np.array_equal(d.view(np.uint32), rd.view(np.uint32))
    ok, info = close(img, ref)
    assert ok, info


def test_instanced_heavy_scene(oracle_lib):
    wl = workloads.heavy_geometry(width=320, height=180, spp=2, dome_size=(128, 64), instanced=True)
    o = oracle_lib.OracleTracer()
    o.set_scene(wl.scene)
    rp, rd = o.trace_primary(wl.camera, wl.width, wl.height, 3)
    ref = o.render(wl.camera, wl.width, wl.height, 0, wl.max_bounces, 1, crop=(100, 60, 164, 124))
    with PathTracer(0) as t:
        t.set_scene(wl.scene)
        inst = t.scene_info()
        p, d = t.trace_primary(wl.camera, wl.width, wl.height, 3)
        img = t.render(wl.camera, wl.width, wl.height, 0, wl.max_bounces, 1)
        t.set_scene(wl.scene.flattened())
        flat = t.scene_info()
    assert np.array_equal(p, rp) and np.array_equal(d.view(np.uint32), rd.view(np.uint32))
    ok, info = close(img[60:124, 100:164], ref[60:124, 100:164])
    assert ok, info
    assert inst["triangles"] == flat["triangles"] == 1_000_480
    assert inst["instances"] == 257 and inst["bottom_levels"] == 5
    assert inst["bvh_bytes"] < flat["bvh_bytes"], (inst, flat)


def test_deforming_instancer_refit_equals_flattened(oracle_lib):
    wl = box_with_instances(3)
    proto = wl.scene.meshes[-1]
    with PathTracer(0) as t:
        t.set_scene(wl.scene)
        rng = np.random.default_rng(5)
        for step in range(2):
            pts = np.asarray(proto.positions, np.float32).reshape(-1, 3)
            pts = (pts * (1.0 + 0.15 * rng.uniform(-1, 1, (len(pts), 1)))).astype(np.float32)
            proto.positions = pts.ravel()
            t.update_instancer_points(0, proto.positions)
            o = oracle_lib.OracleTracer()
            o.set_scene(wl.scene)
            rp, rd = o.trace_primary(wl.camera, 64, 64, step)
            p, d = t.trace_primary(wl.camera, 64, 64, step)
            assert np.array_equal(p, rp) and np.array_equal(d.view(np.uint32), rd.view(np.uint32)), step
            ref = o.render(wl.camera, 64, 64, 0, 8, 2)
            img = t.render(wl.camera, 64, 64, 0, 8, 2)
            ok, info = close(img, ref)
            assert ok, (step, info)
        with pytest.raises(RuntimeError, match="position_count"):
            t.update_instancer_points(0, proto.positions[:-3])
        with pytest.raises(RuntimeError, match="no such instancer"):
            t.update_instancer_points(3, proto.positions)
