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
class Instancer:
    """hdcx_instancer_desc: the mesh `mesh_id` (object space) drawn once per
    transform; transforms is (n, 4, 4) float64, row-vector convention (world =
    [p 1] M), affine."""
    mesh_id: str
    transforms: np.ndarray


@dataclass
class Scene:
    revision: int = 0
    meshes: List[Mesh] = field(default_factory=list)
    materials: List[Material] = field(default_factory=list)
    textures: List[Texture] = field(default_factory=list)
    lights: List[Light] = field(default_factory=list)
    instancers: List[Instancer] = field(default_factory=list)

    def copy(self) -> "Scene":
        return Scene(
            revision=self.revision,
            meshes=[dataclasses.replace(m) for m in self.meshes],
            materials=[m.copy() for m in self.materials],
            textures=[dataclasses.replace(t) for t in self.textures],
            lights=[l.copy() for l in self.lights],
            instancers=[Instancer(i.mesh_id, np.array(i.transforms, dtype=np.float64)) for i in self.instancers],
        )

    def to_desc(self) -> "DescHolder":
        return DescHolder(self)

    def flattened(self) -> "Scene":
        """The scene with every instancer's mesh replaced by its world-space
        copies, as the reference's Hydra mesh adapter flattens an instanced
        mesh (mesh.cpp:955-1004), with the arithmetic include/hdcx.h states for
        hdcx_instancer_desc (the library's own flattening equals it bit for
        bit)."""
        out = self.copy()
        by_id = {inst.mesh_id: inst for inst in self.instancers}
        out.instancers = []
        out.meshes = [flatten_instanced_mesh(m, by_id[m.id].transforms) if m.id in by_id else m for m in out.meshes]
        return out


def _inverse3(m):
    """inverse of the upper 3x3 of m by cofactors / determinant (binary64, the
    operation order of the library's flattening)."""
    a00, a01, a02 = m[0, 0], m[0, 1], m[0, 2]
    a10, a11, a12 = m[1, 0], m[1, 1], m[1, 2]
    a20, a21, a22 = m[2, 0], m[2, 1], m[2, 2]
    c00 = a11 * a22 - a12 * a21
    c01 = a12 * a20 - a10 * a22
    c02 = a10 * a21 - a11 * a20
    det = (a00 * c00 + a01 * c01) + a02 * c02
    return [c00 / det, (a02 * a21 - a01 * a22) / det, (a01 * a12 - a02 * a11) / det,
            c01 / det, (a00 * a22 - a02 * a20) / det, (a02 * a10 - a00 * a12) / det,
            c02 / det, (a01 * a20 - a00 * a21) / det, (a00 * a11 - a01 * a10) / det]


def flatten_instanced_mesh(mesh: "Mesh", transforms) -> "Mesh":
    """World-space copies of `mesh`, one per transform (see Scene.flattened)."""
    T = np.asarray(transforms, dtype=np.float64).reshape(-1, 4, 4)
    P = np.asarray(mesh.positions, dtype=np.float32).reshape(-1, 3).astype(np.float64)
    n = len(P)
    tris = np.asarray(mesh.indices, dtype=np.int64).reshape(-1, 3)
    valid = np.nonzero(np.all(tris < n, axis=1))[0]
    uv = np.asarray(mesh.texcoords, dtype=np.float32).reshape(-1)
    nrm = np.asarray(mesh.normals, dtype=np.float32).reshape(-1)
    corner_normals = len(nrm) // 3
    corners = (3 * valid[:, None] + np.arange(3)[None, :]).reshape(-1)
    has_uv = corners * 2 + 1 < len(uv)
    uvs = np.zeros((len(corners), 2), dtype=np.float32)
    uvs[has_uv, 0] = uv[corners[has_uv] * 2]
    uvs[has_uv, 1] = uv[corners[has_uv] * 2 + 1]
    has_n = corners < corner_normals
    cn = np.zeros((len(corners), 3), dtype=np.float64)
    cn[has_n] = nrm.reshape(-1, 3)[corners[has_n]].astype(np.float64)
    ids = list(mesh.triangle_material_ids)
    tri_ids = [ids[t] if t < len(ids) else mesh.material_id for t in valid]
    positions, indices, texcoords, normals, materials = [], [], [], [], []
    for k, M in enumerate(T):
        if M[0, 3] != 0.0 or M[1, 3] != 0.0 or M[2, 3] != 0.0 or M[3, 3] != 1.0:
            raise ValueError("instancer transforms must be affine")
        w = np.stack([((P[:, 0] * M[0, j] + P[:, 1] * M[1, j]) + P[:, 2] * M[2, j]) + M[3, j] for j in range(3)], 1)
        positions.append(w.astype(np.float32))
        indices.append((tris[valid] + k * n).astype(np.uint32))
        texcoords.append(uvs)
        inv = _inverse3(M)
        v = np.stack([(cn[:, 0] * inv[3 * j] + cn[:, 1] * inv[3 * j + 1]) + cn[:, 2] * inv[3 * j + 2] for j in range(3)], 1)
        length = np.sqrt((v[:, 0] * v[:, 0] + v[:, 1] * v[:, 1]) + v[:, 2] * v[:, 2])
        d = np.where(length > 1e-10, length, 1e-10)
        v = np.where((length <= 1e-12)[:, None], 0.0, v / d[:, None])
        v[~has_n] = 0.0
        normals.append(v.astype(np.float32))
        materials.extend(tri_ids)
    return Mesh(id=mesh.id, positions=np.concatenate(positions).reshape(-1),
                indices=np.concatenate(indices).reshape(-1), texcoords=np.concatenate(texcoords).reshape(-1),
                normals=np.concatenate(normals).reshape(-1), material_id=mesh.material_id,
                triangle_material_ids=materials, display_color=mesh.display_color)


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

        mesh_index = {m.id: i for i, m in enumerate(scene.meshes)}
        instancers = (_abi.InstancerDesc * max(1, len(scene.instancers)))()
        for i, inst in enumerate(scene.instancers):
            t = np.ascontiguousarray(np.asarray(inst.transforms, dtype=np.float64).reshape(-1))
            keep.append(t)
            instancers[i].mesh_index = mesh_index[inst.mesh_id]
            instancers[i].transforms = t.ctypes.data_as(C.POINTER(C.c_double))
            instancers[i].instance_count = t.size // 16
        self.instancers = instancers
        self.instancer_count = len(scene.instancers)
        keep.extend([meshes, materials, textures, lights, instancers])
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
