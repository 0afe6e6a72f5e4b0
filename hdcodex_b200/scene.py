"""Scene snapshot types: Python mirrors of the reference's scene ABI.

``Mesh``, ``Material``, ``Texture``, ``Light`` and ``Scene`` correspond field
for field to SceneMesh, SceneMaterial (its path-closure members), SceneTexture,
SceneLight and SceneSnapshot (include/hdcodex/core/versioned_scene.h:17-274),
with the same defaults, so scenes read like the reference's tests
(tests/path_tracer_tests.cpp). ``Scene.to_desc()`` marshals a snapshot into the
C structs of include/hdcx.h; the returned holder keeps every buffer alive.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

from . import _abi

# SceneLightType / DomeTextureFormat / DiffuseModel values.
DOME, RECT, DISK, SPHERE, CYLINDER, DISTANT = range(6)
AUTOMATIC, LATLONG, MIRRORED_BALL, ANGULAR, CUBEMAP_VERTICAL_CROSS = range(5)
LAMBERT, OREN_NAYAR, BURLEY, OREN_NAYAR_ENERGY_COMPENSATED = range(4)


def _material_defaults():
    return {n: (list(d) if isinstance(d, tuple) else d) for n, _, d in _abi.MATERIAL_FIELDS}


def _light_defaults():
    return {n: (list(d) if isinstance(d, tuple) else d) for n, _, d in _abi.LIGHT_FIELDS}


@dataclass
class Mesh:
    id: str
    positions: Sequence[float] = ()
    indices: Sequence[int] = ()
    texcoords: Sequence[float] = ()
    normals: Sequence[float] = ()
    material_id: str = ""
    triangle_material_ids: Sequence[str] = ()
    display_color: Sequence[float] = (0.5, 0.5, 0.5)


class _FieldBag:
    """Attribute bag whose fields and defaults come from an ABI field table."""

    _defaults = staticmethod(dict)

    def __init__(self, **kwargs):
        values = self._defaults()
        for key, value in kwargs.items():
            if key not in values:
                raise TypeError(f"{type(self).__name__} has no field {key!r}")
            values[key] = value
        self.__dict__.update(values)

    def __setattr__(self, key, value):
        if key not in self.__dict__:
            raise AttributeError(f"{type(self).__name__} has no field {key!r}")
        self.__dict__[key] = value

    def copy(self, **changes):
        values = dict(self.__dict__)
        values.update(changes)
        return type(self)(**values)

    def __repr__(self):
        return f"{type(self).__name__}(id={self.__dict__.get('id')!r})"


class Material(_FieldBag):
    """SceneMaterial's compact closure ABI (versioned_scene.h:117-188)."""

    _defaults = staticmethod(_material_defaults)


class Light(_FieldBag):
    """SceneLight (versioned_scene.h:225-266)."""

    _defaults = staticmethod(_light_defaults)


@dataclass
class Texture:
    id: str
    source_path: str = ""
    udim_set_id: str = ""
    udim_tile: int = 0
    width: int = 0
    height: int = 0
    srgb: bool = False
    rgba: Optional[Sequence[int]] = None
    rgba_float: Optional[Sequence[float]] = None


@dataclass
class Scene:
    revision: int = 0
    meshes: List[Mesh] = field(default_factory=list)
    materials: List[Material] = field(default_factory=list)
    textures: List[Texture] = field(default_factory=list)
    lights: List[Light] = field(default_factory=list)

    def copy(self) -> "Scene":
        return Scene(
            revision=self.revision,
            meshes=[dataclasses.replace(m) for m in self.meshes],
            materials=[m.copy() for m in self.materials],
            textures=[dataclasses.replace(t) for t in self.textures],
            lights=[l.copy() for l in self.lights],
        )

    def to_desc(self) -> "DescHolder":
        return DescHolder(self)


def _b(s: Optional[str]) -> Optional[bytes]:
    return s.encode() if s else None


class DescHolder:
    """Owns the C structs and arrays of one marshalled snapshot."""

    def __init__(self, scene: Scene):
        keep = []
        self._keep = keep

        def farr(values, dtype=np.float32):
            if values is None or len(values) == 0:
                return None, 0
            a = np.ascontiguousarray(np.asarray(values, dtype=dtype).reshape(-1))
            keep.append(a)
            ctype = {np.float32: C.c_float, np.uint32: C.c_uint32, np.uint8: C.c_uint8}[dtype]
            return a.ctypes.data_as(C.POINTER(ctype)), a.size

        meshes = (_abi.MeshDesc * max(1, len(scene.meshes)))()
        for i, m in enumerate(scene.meshes):
            d = meshes[i]
            d.id = _b(m.id)
            d.positions, d.position_count = farr(m.positions)
            d.indices, d.index_count = farr(m.indices, np.uint32)
            d.texcoords, d.texcoord_count = farr(m.texcoords)
            d.normals, d.normal_count = farr(m.normals)
            d.material_id = _b(m.material_id)
            if m.triangle_material_ids:
                ids = (C.c_char_p * len(m.triangle_material_ids))(
                    *[(s.encode() if s else b"") for s in m.triangle_material_ids])
                keep.append(ids)
                d.triangle_material_ids = ids
                d.triangle_material_id_count = len(m.triangle_material_ids)
            d.display_color = _abi.F3(*m.display_color)

        materials = (_abi.MaterialDesc * max(1, len(scene.materials)))()
        for i, m in enumerate(scene.materials):
            d = materials[i]
            for name, ctype, _ in _abi.MATERIAL_FIELDS:
                value = getattr(m, name)
                if ctype is C.c_char_p:
                    setattr(d, name, _b(value))
                elif ctype is _abi.F3:
                    setattr(d, name, _abi.F3(*value))
                else:
                    setattr(d, name, int(value) if ctype in (C.c_int32, C.c_uint32) else float(value))

        textures = (_abi.TextureDesc * max(1, len(scene.textures)))()
        for i, t in enumerate(scene.textures):
            d = textures[i]
            d.id = _b(t.id)
            d.udim_set_id = _b(t.udim_set_id)
            d.udim_tile = t.udim_tile
            d.width = t.width
            d.height = t.height
            d.srgb = 1 if t.srgb else 0
            if t.rgba is not None and len(t.rgba):
                d.rgba, d.rgba_count = farr(t.rgba, np.uint8)
            if t.rgba_float is not None and len(t.rgba_float):
                d.rgba_float, d.rgba_float_count = farr(t.rgba_float)

        lights = (_abi.LightDesc * max(1, len(scene.lights)))()
        for i, l in enumerate(scene.lights):
            d = lights[i]
            for name, ctype, _ in _abi.LIGHT_FIELDS:
                value = getattr(l, name)
                if ctype is C.c_char_p:
                    setattr(d, name, _b(value))
                elif ctype is _abi.F3:
                    setattr(d, name, _abi.F3(*value))
                else:
                    setattr(d, name, int(value) if ctype in (C.c_int32, C.c_uint32) else float(value))

        keep.extend([meshes, materials, textures, lights])
        self.desc = _abi.SceneDesc(
            revision=scene.revision,
            meshes=meshes, mesh_count=len(scene.meshes),
            materials=materials, material_count=len(scene.materials),
            textures=textures, texture_count=len(scene.textures),
            lights=lights, light_count=len(scene.lights),
        )

    def pointer(self):
        return C.byref(self.desc)


def camera(origin, lower_left, horizontal, vertical) -> _abi.Camera:
    """PathTracerCamera (vulkan_path_tracer.h:16-23)."""
    return _abi.Camera(_abi.F3(*origin), _abi.F3(*lower_left), _abi.F3(*horizontal),
                       _abi.F3(*vertical))
