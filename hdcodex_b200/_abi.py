"""ctypes mirrors of the C ABI structs in include/hdcx.h.

The field tables below are the single Python statement of the scene ABI: the
ctypes structures are generated from them and the dataclasses in scene.py take
their defaults from them. Defaults are those of the reference's scene ABI
(include/hdcodex/core/versioned_scene.h:17-34 SceneMesh, :121-188
SceneMaterial, :225-266 SceneLight).
"""
from __future__ import annotations

import ctypes as C

F3 = C.c_float * 3

# (name, ctype, default). Texture ids are strings (c_char_p) defaulting to "".
MATERIAL_FIELDS = [
    ("id", C.c_char_p, ""),
    ("base_color", F3, (0.8, 0.8, 0.8)),
    ("base_color_texture_scale", F3, (1.0, 1.0, 1.0)),
    ("base_color_texture_bias", F3, (0.0, 0.0, 0.0)),
    ("base_color_texture_channel", C.c_int32, -1),
    ("emission", F3, (0.0, 0.0, 0.0)),
    ("transmission_color", F3, (1.0, 1.0, 1.0)),
    ("transmission_scatter", F3, (0.0, 0.0, 0.0)),
    ("specular_color", F3, (1.0, 1.0, 1.0)),
    ("coat_color", F3, (1.0, 1.0, 1.0)),
    ("sheen_color", F3, (1.0, 1.0, 1.0)),
    ("translucent_color", F3, (1.0, 1.0, 1.0)),
    ("subsurface_color", F3, (0.8, 0.8, 0.8)),
    ("subsurface_radius", F3, (1.0, 0.2, 0.1)),
    ("diffuse_model", C.c_uint32, 0),
    ("diffuse_weight", C.c_float, 1.0),
    ("diffuse_roughness", C.c_float, 0.0),
    ("metalness", C.c_float, 0.0),
    ("roughness", C.c_float, 0.5),
    ("roughness_v", C.c_float, 0.5),
    ("opacity", C.c_float, 1.0),
    ("emission_weight", C.c_float, 0.0),
    ("transmission", C.c_float, 0.0),
    ("transmission_depth", C.c_float, 0.0),
    ("transmission_scatter_anisotropy", C.c_float, 0.0),
    ("transmission_dispersion_scale", C.c_float, 0.0),
    ("transmission_dispersion_abbe_number", C.c_float, 20.0),
    ("index_of_refraction", C.c_float, 1.5),
    ("specular_weight", C.c_float, 1.0),
    ("coat", C.c_float, 0.0),
    ("coat_roughness", C.c_float, 0.1),
    ("coat_roughness_v", C.c_float, 0.1),
    ("coat_index_of_refraction", C.c_float, 1.5),
    ("sheen", C.c_float, 0.0),
    ("sheen_roughness", C.c_float, 0.3),
    ("sheen_mode", C.c_uint32, 0),
    ("translucent_weight", C.c_float, 0.0),
    ("subsurface", C.c_float, 0.0),
    ("subsurface_scale", C.c_float, 1.0),
    ("subsurface_scatter_anisotropy", C.c_float, 0.0),
    ("thin_walled", C.c_int32, False),
    ("normal_texture_flip_y", C.c_int32, False),
    ("normal_texture_scale", C.c_float, 1.0),
    ("base_color_texture", C.c_char_p, ""),
    ("metalness_texture", C.c_char_p, ""),
    ("roughness_texture", C.c_char_p, ""),
    ("diffuse_weight_texture", C.c_char_p, ""),
    ("diffuse_roughness_texture", C.c_char_p, ""),
    ("emission_texture", C.c_char_p, ""),
    ("opacity_texture", C.c_char_p, ""),
    ("normal_texture", C.c_char_p, ""),
    ("transmission_texture", C.c_char_p, ""),
    ("specular_texture", C.c_char_p, ""),
    ("specular_color_texture", C.c_char_p, ""),
    ("coat_texture", C.c_char_p, ""),
    ("coat_color_texture", C.c_char_p, ""),
    ("coat_roughness_texture", C.c_char_p, ""),
    ("sheen_texture", C.c_char_p, ""),
    ("sheen_color_texture", C.c_char_p, ""),
    ("sheen_roughness_texture", C.c_char_p, ""),
    ("translucent_weight_texture", C.c_char_p, ""),
    ("translucent_color_texture", C.c_char_p, ""),
    ("subsurface_texture", C.c_char_p, ""),
    ("subsurface_color_texture", C.c_char_p, ""),
    ("subsurface_radius_texture", C.c_char_p, ""),
]

LIGHT_FIELDS = [
    ("id", C.c_char_p, ""),
    ("type", C.c_uint32, 0),
    ("visible", C.c_int32, True),
    ("color", F3, (1.0, 1.0, 1.0)),
    ("temperature_color", F3, (1.0, 1.0, 1.0)),
    ("intensity", C.c_float, 1.0),
    ("exposure", C.c_float, 0.0),
    ("diffuse", C.c_float, 1.0),
    ("specular", C.c_float, 1.0),
    ("normalize", C.c_int32, False),
    ("texture", C.c_char_p, ""),
    ("texture_format", C.c_uint32, 0),
    ("basis_x", F3, (1.0, 0.0, 0.0)),
    ("basis_y", F3, (0.0, 1.0, 0.0)),
    ("basis_z", F3, (0.0, 0.0, 1.0)),
    ("position", F3, (0.0, 0.0, 0.0)),
    ("axis_u", F3, (1.0, 0.0, 0.0)),
    ("axis_v", F3, (0.0, 1.0, 0.0)),
    ("width", C.c_float, 1.0),
    ("height", C.c_float, 1.0),
    ("radius", C.c_float, 0.5),
    ("length", C.c_float, 1.0),
    ("angle", C.c_float, 0.53),
    ("area", C.c_float, 1.0),
    ("shaping_focus", C.c_float, 0.0),
    ("shaping_focus_tint", F3, (0.0, 0.0, 0.0)),
    ("shaping_cone_angle", C.c_float, 180.0),
    ("shaping_cone_softness", C.c_float, 0.0),
    ("shadow_enable", C.c_int32, True),
    ("shadow_color", F3, (0.0, 0.0, 0.0)),
    ("shadow_distance", C.c_float, -1.0),
    ("shadow_falloff", C.c_float, -1.0),
    ("shadow_falloff_gamma", C.c_float, 1.0),
]


class Camera(C.Structure):
    _fields_ = [("origin", F3), ("lower_left", F3), ("horizontal", F3), ("vertical", F3)]


class MeshDesc(C.Structure):
    _fields_ = [
        ("id", C.c_char_p),
        ("positions", C.POINTER(C.c_float)),
        ("position_count", C.c_uint64),
        ("indices", C.POINTER(C.c_uint32)),
        ("index_count", C.c_uint64),
        ("texcoords", C.POINTER(C.c_float)),
        ("texcoord_count", C.c_uint64),
        ("normals", C.POINTER(C.c_float)),
        ("normal_count", C.c_uint64),
        ("material_id", C.c_char_p),
        ("triangle_material_ids", C.POINTER(C.c_char_p)),
        ("triangle_material_id_count", C.c_uint64),
        ("display_color", F3),
    ]


class MaterialDesc(C.Structure):
    _fields_ = [(n, t) for n, t, _ in MATERIAL_FIELDS]


class TextureDesc(C.Structure):
    _fields_ = [
        ("id", C.c_char_p),
        ("udim_set_id", C.c_char_p),
        ("udim_tile", C.c_uint32),
        ("width", C.c_uint32),
        ("height", C.c_uint32),
        ("srgb", C.c_int32),
        ("rgba", C.POINTER(C.c_uint8)),
        ("rgba_count", C.c_uint64),
        ("rgba_float", C.POINTER(C.c_float)),
        ("rgba_float_count", C.c_uint64),
    ]


class LightDesc(C.Structure):
    _fields_ = [(n, t) for n, t, _ in LIGHT_FIELDS]


class SceneDesc(C.Structure):
    _fields_ = [
        ("revision", C.c_uint64),
        ("meshes", C.POINTER(MeshDesc)),
        ("mesh_count", C.c_uint64),
        ("materials", C.POINTER(MaterialDesc)),
        ("material_count", C.c_uint64),
        ("textures", C.POINTER(TextureDesc)),
        ("texture_count", C.c_uint64),
        ("lights", C.POINTER(LightDesc)),
        ("light_count", C.c_uint64),
    ]


class PackedTexture(C.Structure):
    _fields_ = [
        ("width", C.c_uint32),
        ("height", C.c_uint32),
        ("format", C.c_uint32),
        ("reserved", C.c_uint32),
        ("texels", C.c_void_p),
    ]


class PackedScene(C.Structure):
    _fields_ = [
        ("vertex_count", C.c_uint32),
        ("triangle_count", C.c_uint32),
        ("material_count", C.c_uint32),
        ("light_count", C.c_uint32),
        ("texture_count", C.c_uint32),
        ("opaque", C.c_uint32),
        ("vertices", C.POINTER(C.c_float)),
        ("indices", C.POINTER(C.c_uint32)),
        ("triangle_materials", C.POINTER(C.c_uint32)),
        ("texcoords", C.POINTER(C.c_float)),
        ("normals", C.POINTER(C.c_float)),
        ("materials", C.c_void_p),
        ("lights", C.c_void_p),
        ("emissive", C.POINTER(C.c_float)),
        ("textures", C.POINTER(PackedTexture)),
    ]


class RenderStats(C.Structure):
    _fields_ = [
        ("spectral_paths", C.c_uint64),
        ("extension_rays", C.c_uint64),
        ("shadow_rays", C.c_uint64),
        ("subsurface_rays", C.c_uint64),
        ("render_ms", C.c_double),
        ("extend_ms", C.c_double),
        ("shade_ms", C.c_double),
        ("shadow_ms", C.c_double),
        ("waves", C.c_uint32),
        ("extend_launches", C.c_uint32),
        ("kernel_launches", C.c_uint64),
        ("extension_node_visits", C.c_uint64),
        ("extension_triangle_tests", C.c_uint64),
        ("shadow_node_visits", C.c_uint64),
        ("shadow_triangle_tests", C.c_uint64),
    ]


class NrcConfig(C.Structure):
    """hdcx_nrc_config."""
    _fields_ = [
        ("log2_table_size", C.c_uint32),
        ("base_resolution", C.c_uint32),
        ("finest_resolution", C.c_uint32),
        ("learning_rate", C.c_float),
        ("beta1", C.c_float),
        ("beta2", C.c_float),
        ("epsilon", C.c_float),
        ("seed", C.c_uint32),
    ]


class BatchJob(C.Structure):
    """hdcx_batch_job: one job of hdcx_render_batch."""
    _fields_ = [
        ("tracer", C.c_void_p),
        ("camera", Camera),
        ("width", C.c_uint32),
        ("height", C.c_uint32),
        ("sample_index", C.c_uint32),
        ("max_bounces", C.c_uint32),
        ("sample_count", C.c_uint32),
        ("rgba_out", C.c_void_p),
        ("written", C.c_int32),
        ("status", C.c_int32),
        ("render_ms", C.c_double),
    ]


class Tuning(C.Structure):
    """hdcx_tuning."""
    _fields_ = [
        ("wave_paths", C.c_uint64),
        ("trace_blocks_per_sm", C.c_uint32),
        ("shade_blocks_per_sm", C.c_uint32),
        ("milliseconds", C.c_double),
        ("default_milliseconds", C.c_double),
        ("candidates", C.c_uint32),
        ("sort_hits", C.c_uint32),
        ("sort_rays", C.c_uint32),
    ]


class InstancerDesc(C.Structure):
    _fields_ = [
        ("mesh_index", C.c_uint64),
        ("transforms", C.POINTER(C.c_double)),
        ("instance_count", C.c_uint64),
    ]


class SceneInfo(C.Structure):
    _fields_ = [
        ("triangles", C.c_uint64),
        ("instances", C.c_uint64),
        ("bottom_levels", C.c_uint64),
        ("bvh_bytes", C.c_uint64),
        ("scene_bytes", C.c_uint64),
        ("build_ms", C.c_double),
        ("bvh_build_ms", C.c_double),
    ]


STRUCTS_IN_ABI_ORDER = [
    Camera, MeshDesc, MaterialDesc, TextureDesc, LightDesc, SceneDesc, PackedTexture, PackedScene,
    RenderStats, BatchJob, NrcConfig, Tuning, InstancerDesc, SceneInfo,
]

GPU_MATERIAL_BYTES = 368
GPU_LIGHT_BYTES = 224
MISSING_TEXTURE = 0xFFFFFFFF
