"""Host packing: the product's SceneSnapshot packing equals the oracle's
restatement of the reference's BuildScene (vulkan_path_tracer.cpp:2604-2993)
byte for byte - GpuMaterial/GpuLight records, flattened geometry, material
indices, UDIM descriptor words, dome importance CDFs and the FP64 emissive
CDF."""
import numpy as np
import pytest

import ref_scenes as R
from hdcodex_b200 import pack_scene, workloads
from hdcodex_b200.scene import DOME, LATLONG, Light, Material, Mesh, Scene, Texture

VARIANTS = ["base", "oren_nayar", "udim", "authored_normals", "glossy", "coated", "subsurface", "cutout",
            "translucent", "thin_walled", "dispersive", "fallback"]


def assert_same_packing(a: dict, b: dict):
    for key in ("vertex_count", "triangle_count", "material_count", "light_count", "texture_count", "opaque"):
        assert a[key] == b[key], key
    for key in ("vertices", "indices", "triangle_materials", "texcoords", "normals", "materials", "lights",
                "emissive"):
        assert a[key].tobytes() == b[key].tobytes(), key
    assert len(a["textures"]) == len(b["textures"])
    for ta, tb in zip(a["textures"], b["textures"]):
        assert ta[:3] == tb[:3]
        assert ta[3].tobytes() == tb[3].tobytes()


def oracle_packing(oracle_lib, scene):
    t = oracle_lib.OracleTracer()
    t.set_scene(scene)
    return t.packed()


@pytest.mark.parametrize("name", VARIANTS)
def test_reference_scene_packing_matches_oracle(oracle_lib, hdcx_lib, name):
    scene = R.variant(name)
    assert_same_packing(pack_scene(scene), oracle_packing(oracle_lib, scene))


def test_selection_and_mesh_light_scenes(oracle_lib, hdcx_lib):
    for scene in (R.selection_scene(), R.mesh_light_scene(1.0), R.mesh_light_scene(0.0)):
        assert_same_packing(pack_scene(scene), oracle_packing(oracle_lib, scene))


def test_closed_box_packing(oracle_lib, hdcx_lib):
    for quad in (False, True):
        scene = workloads.closed_box(emissive_quad=quad).scene
        assert_same_packing(pack_scene(scene), oracle_packing(oracle_lib, scene))


def test_packing_rules(hdcx_lib):
    """Reference ordering rules: default material 0, materials in snapshot
    order, display-colour materials deduplicated, subsets resolve per
    triangle, out-of-range triangles dropped, 64-light cap, UDIM words."""
    s = Scene()
    s.materials = [Material(id="/a", base_color=[0.1, 0.2, 0.3]), Material(id="/b", emission=[1.0, 0.0, 0.0],
                                                                            emission_weight=2.0)]
    s.meshes = [
        Mesh(id="/m0", positions=[0, 0, 0, 1, 0, 0, 0, 1, 0, 1, 1, 0], indices=[0, 1, 2, 1, 3, 2, 0, 1, 9],
             material_id="/a", triangle_material_ids=["/a", "/b", "/missing"]),
        Mesh(id="/m1", positions=[0, 0, 1, 1, 0, 1, 0, 1, 1], indices=[0, 1, 2], display_color=[2.0, 0.5, -1.0]),
        Mesh(id="/m2", positions=[0, 0, 2, 1, 0, 2, 0, 1, 2], indices=[0, 1, 2], display_color=[1.0, 0.5, 0.0]),
    ]
    s.textures = [Texture(id="u#1", udim_set_id="u", udim_tile=1001, width=1, height=1, rgba=[1, 2, 3, 4]),
                  Texture(id="u#3", udim_set_id="u", udim_tile=1003, width=1, height=1, rgba=[1, 2, 3, 4]),
                  Texture(id="bad", width=2, height=2, rgba=[0, 0, 0, 0])]
    s.lights = [Light(id=f"/l{i}", intensity=0.0) for i in range(70)]
    p = pack_scene(s)
    assert p["triangle_count"] == 4  # the index-9 triangle is dropped
    assert p["triangle_materials"].tolist() == [1, 2, 3, 3]  # /a, /b, clamped display colour twice
    assert p["material_count"] == 4
    assert p["light_count"] == 64
    assert p["texture_count"] == 2
    # UDIM word: flag | present tiles (1001, 1003) << 8 | base 0
    s.materials[0].base_color_texture = "u"
    mats = pack_scene(s)["materials"].view(np.uint32).reshape(-1, 92)
    assert mats[1, 68] == 0x80000000 | (0b101 << 8) | 0
    # Emissive CDF: only the /b triangle emits, so the CDF steps to 1 there.
    e = p["emissive"].reshape(-1, 4)
    assert e[1, 0] == 1.0 and e[-1, 0] == 1.0 and e[0, 0] == 0.0 and e[1, 1] > 0


def test_dome_importance_map(oracle_lib, hdcx_lib):
    rng = np.random.default_rng(3)
    w, h = 16, 8
    rgba = rng.lognormal(0.0, 1.0, size=(h, w, 4)).astype(np.float32)
    rgba[..., 3] = 1
    s = R.base_scene()
    s.textures.append(Texture(id="env#hdr", width=w, height=h, rgba_float=rgba.ravel()))
    s.lights[0].texture = "env#hdr"
    s.lights[0].texture_format = LATLONG
    p = pack_scene(s)
    assert_same_packing(p, oracle_packing(oracle_lib, s))
    imp = p["textures"][-1]
    assert imp[:3] == (w, h, 2)
    m = imp[3].reshape(h, w, 4)
    assert np.all(m[:, -1, 0] == 1.0) and m[-1, 0, 1] == 1.0
    assert np.all(np.diff(m[:, :, 0], axis=1) >= 0) and np.all(np.diff(m[:, 0, 1]) >= 0)
    # pdf integrates to 1 over the sphere: sum(pdf * solid angle) = 1.
    v0 = np.arange(h) / h
    v1 = (np.arange(h) + 1) / h
    solid = (2 * np.pi / w) * np.abs(np.cos(np.pi * (1 - v1)) - np.cos(np.pi * (1 - v0)))
    assert (m[:, :, 2] * solid[:, None]).sum() == pytest.approx(1.0, rel=1e-5)


@pytest.mark.parametrize("seed", range(12))
def test_random_scene_packing_matches_oracle(oracle_lib, hdcx_lib, seed):
    """The random material, light and texture scenes of the shader fuzz tests
    (ref_scenes.fuzz_box, fuzz_lights_box, fuzz_textured) pack byte for byte
    as the oracle's restatement of BuildScene packs them."""
    for scene in (R.fuzz_box(seed).scene, R.fuzz_lights_box(seed).scene, R.fuzz_textured(seed)):
        assert_same_packing(pack_scene(scene), oracle_packing(oracle_lib, scene))
