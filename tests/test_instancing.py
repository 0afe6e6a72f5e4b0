"""Instancers (hdcx_instancer_desc), host side: the library's flattening of an
instanced mesh equals the documented one (Scene.flattened, numpy binary64)
bit for bit, so a two-level scene packs exactly like its flattened snapshot.
No GPU needed; the GPU tests (test_gpu_instancing.py) render both forms."""
import numpy as np
import pytest

import ref_scenes as R
from hdcodex_b200 import Instancer, Mesh, pack_scene, workloads


def random_affine(rng, translate=5.0):
    A = rng.normal(size=(3, 3))
    A += np.eye(3) * 2.0  # well conditioned: scale, rotation and shear
    M = np.zeros((4, 4))
    M[:3, :3] = A
    M[3, :3] = rng.uniform(-translate, translate, 3)
    M[3, 3] = 1.0
    return M


def instanced_scene(seed=0, instances=5, invalid=True):
    rng = np.random.default_rng(seed)
    scene = R.base_scene()
    v, f = workloads._icosphere(1)
    v = v.astype(np.float32)
    tris = f.astype(np.int64)
    if invalid:  # a triangle with an out-of-range index is dropped by the flattening
        tris = np.vstack([tris, [[0, 1, len(v) + 3]]])
    corners = tris.size
    normals = rng.normal(size=(corners, 3)).astype(np.float32)
    normals[::7] = 0.0  # zero normals stay zero
    uvs = rng.uniform(0, 1, (corners - 3, 2)).astype(np.float32)  # the last corners have no uv
    ids = [scene.materials[0].id if t % 3 else "" for t in range(len(tris) - 2)]
    proto = Mesh(id="/proto", positions=v.ravel(), indices=tris.astype(np.uint32).ravel(), texcoords=uvs.ravel(),
                 normals=normals.ravel(), material_id=scene.materials[0].id, triangle_material_ids=ids)
    scene.meshes.insert(0, proto)
    scene.instancers = [Instancer("/proto", np.array([random_affine(rng) for _ in range(instances)]))]
    return scene


@pytest.mark.parametrize("seed", range(6))
def test_instanced_packing_equals_flattened_packing(hdcx_lib, seed):
    scene = instanced_scene(seed)
    a = pack_scene(scene)
    b = pack_scene(scene.flattened())
    for key in ("vertex_count", "triangle_count", "material_count", "light_count", "opaque"):
        assert a[key] == b[key], key
    for key in ("vertices", "indices", "triangle_materials", "texcoords", "normals", "materials", "lights", "emissive"):
        assert a[key].tobytes() == b[key].tobytes(), key


def test_flattening_follows_the_adapter_layout(hdcx_lib):
    scene = instanced_scene(1, instances=3)
    flat = scene.flattened()
    proto = scene.meshes[0]
    m = flat.meshes[0]
    n = len(proto.positions) // 3
    valid = len(proto.indices) // 3 - 1  # one invalid triangle dropped
    assert len(m.positions) == 3 * n * 3
    assert len(m.indices) == 3 * valid * 3
    assert m.indices.max() < 3 * n and m.indices[3 * valid] == m.indices[0] + n  # instance-major, vertex base per instance
    assert len(m.triangle_material_ids) == 3 * valid
    # Identity transform: world = object exactly, normals normalised.
    ident = scene.copy()
    ident.instancers = [Instancer("/proto", np.eye(4)[None])]
    f = ident.flattened().meshes[0]
    assert np.array_equal(f.positions, np.asarray(proto.positions, np.float32))
    lengths = np.linalg.norm(f.normals.reshape(-1, 3).astype(np.float64), axis=1)
    assert np.all((np.abs(lengths - 1) < 1e-6) | (lengths == 0))


def test_non_affine_transform_is_rejected(hdcx_lib):
    scene = instanced_scene(2, instances=1)
    scene.instancers[0].transforms[0, 0, 3] = 0.5
    with pytest.raises(RuntimeError):
        pack_scene(scene)
    with pytest.raises(ValueError):
        scene.flattened()


def test_instanced_heavy_workload_has_the_config_shape():
    wl = workloads.heavy_geometry(width=64, height=36, spp=1, dome_size=(16, 8), instanced=True)
    flat = wl.scene.flattened()
    assert workloads.triangle_count(flat) == 1_000_480
    assert sum(len(i.transforms) for i in wl.scene.instancers) == 256
