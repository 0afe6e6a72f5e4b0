"""Seeded synthetic scenes of the benchmark configurations.

* ``closed_box``  - 5 Lambert walls + 2 inner boxes (34 triangles), a ceiling
  rect light of colour (17, 12, 4); 256x256, 16 spp, 8 bounces.
* ``heavy_geometry`` - 256 noise-displaced icospheres (level 3, 1,280
  triangles each) on a 581x581-vertex heightfield: 1,000,480 triangles;
  per-triangle materials drawn from Lambert, GGX dielectric (roughness
  U[0.05, 0.8], IOR 1.5) and GGX conductor through per-triangle subsets; a
  2048x1024 RGBA32F lat-long dome with log-normal luminance (sigma 2) and
  three Gaussian hotspots; 1920x1080, 64 spp, 8 bounces.
* ``spectral_stress`` - a ~200k-triangle sphere, torus and plinth with a
  dispersive dielectric (Abbe 20-60), Beer absorption, interior scattering,
  subsurface random walk and opacity-cutout leaves; 1280x720, 256 spp.

All geometry is fp32, flattened into world space as hdCodex's mesh adapter
does for instancers (src/hydra/mesh.cpp:955-1004). Every generator is a pure
function of its seed.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from .scene import DOME, LATLONG, RECT, Light, Material, Mesh, Scene, Texture, camera


@dataclass
class Workload:
    name: str
    scene: Scene
    camera: object
    width: int
    height: int
    spp: int
    max_bounces: int

    @property
    def spectral_paths(self) -> int:
        return self.width * self.height * self.spp * 3


def look_at_camera(origin, target, up, vfov_deg, aspect):
    """PathTracerCamera of a pinhole at `origin` looking at `target`."""
    o = np.asarray(origin, dtype=np.float64)
    w = o - np.asarray(target, dtype=np.float64)
    w /= np.linalg.norm(w)
    u = np.cross(np.asarray(up, dtype=np.float64), w)
    u /= np.linalg.norm(u)
    v = np.cross(w, u)
    half_h = math.tan(math.radians(vfov_deg) / 2.0)
    half_w = aspect * half_h
    lower_left = o - half_w * u - half_h * v - w
    return camera(o.tolist(), lower_left.tolist(), (2 * half_w * u).tolist(), (2 * half_h * v).tolist())


def _quad(p0, p1, p2, p3):
    return [p0, p1, p2, p3], [0, 1, 2, 0, 2, 3]


def _box_mesh(lo, hi):
    x0, y0, z0 = lo
    x1, y1, z1 = hi
    v = [(x0, y0, z0), (x1, y0, z0), (x1, y1, z0), (x0, y1, z0),
         (x0, y0, z1), (x1, y0, z1), (x1, y1, z1), (x0, y1, z1)]
    f = [0, 2, 1, 0, 3, 2, 4, 5, 6, 4, 6, 7, 0, 1, 5, 0, 5, 4,
         3, 7, 6, 3, 6, 2, 0, 4, 7, 0, 7, 3, 1, 2, 6, 1, 6, 5]
    return v, f


def closed_box(width=256, height=256, spp=16, max_bounces=8, emissive_quad=False) -> Workload:
    """5 walls (10 triangles) + 2 axis-aligned boxes (24 triangles), one quad light."""
    s = Scene(revision=1)
    s.materials = [
        Material(id="/white", base_color=[0.73, 0.73, 0.73], specular_weight=0.0),
        Material(id="/red", base_color=[0.63, 0.065, 0.05], specular_weight=0.0),
        Material(id="/green", base_color=[0.14, 0.45, 0.09], specular_weight=0.0),
    ]
    walls = [
        ("/floor", _quad((0, 0, 0), (1, 0, 0), (1, 0, 1), (0, 0, 1)), "/white"),
        ("/ceiling", _quad((0, 1, 0), (0, 1, 1), (1, 1, 1), (1, 1, 0)), "/white"),
        ("/back", _quad((0, 0, 0), (0, 1, 0), (1, 1, 0), (1, 0, 0)), "/white"),
        ("/left", _quad((0, 0, 0), (0, 0, 1), (0, 1, 1), (0, 1, 0)), "/red"),
        ("/right", _quad((1, 0, 0), (1, 1, 0), (1, 1, 1), (1, 0, 1)), "/green"),
    ]
    for name, (verts, idx), mat in walls:
        s.meshes.append(Mesh(id=name, positions=np.asarray(verts, np.float32).ravel().tolist(), indices=idx,
                             material_id=mat))
    for name, lo, hi in (("/tall", (0.18, 0.0, 0.2), (0.45, 0.62, 0.48)),
                         ("/short", (0.56, 0.0, 0.52), (0.82, 0.3, 0.8))):
        verts, idx = _box_mesh(lo, hi)
        s.meshes.append(Mesh(id=name, positions=np.asarray(verts, np.float32).ravel().tolist(), indices=idx,
                             material_id="/white"))
    if emissive_quad:
        s.materials.append(Material(id="/lamp", base_color=[0.0, 0.0, 0.0], emission=[17.0, 12.0, 4.0],
                                    emission_weight=1.0, specular_weight=0.0))
        verts, idx = _quad((0.375, 0.998, 0.375), (0.625, 0.998, 0.375), (0.625, 0.998, 0.625),
                           (0.375, 0.998, 0.625))
        s.meshes.append(Mesh(id="/lamp", positions=np.asarray(verts, np.float32).ravel().tolist(), indices=idx,
                             material_id="/lamp"))
        s.lights = []
    else:
        s.lights = [Light(id="/ceilingLight", type=RECT, color=[17.0, 12.0, 4.0], intensity=1.0,
                          normalize=False, position=[0.5, 0.998, 0.5], basis_x=[1.0, 0.0, 0.0],
                          basis_y=[0.0, 0.0, 1.0], basis_z=[0.0, 1.0, 0.0], axis_u=[0.25, 0.0, 0.0],
                          axis_v=[0.0, 0.0, 0.25], width=0.25, height=0.25, area=0.0625)]
    cam = look_at_camera((0.5, 0.5, 2.1), (0.5, 0.5, 0.0), (0.0, 1.0, 0.0), 38.0, width / height)
    return Workload("closed-box-34tri", s, cam, width, height, spp, max_bounces)


def _icosphere(level: int):
    t = (1.0 + math.sqrt(5.0)) / 2.0
    verts = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
             (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    verts = [np.asarray(v, np.float64) / np.linalg.norm(v) for v in verts]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
             (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5),
             (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(level):
        cache = {}
        out = []

        def mid(a, b):
            key = (min(a, b), max(a, b))
            if key not in cache:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                cache[key] = len(verts) - 1
            return cache[key]

        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            out += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = out
    return np.asarray(verts, np.float64), np.asarray(faces, np.uint32)


def _noise3(p: np.ndarray, rng: np.random.Generator, octaves: int = 4) -> np.ndarray:
    """Sum of seeded random sinusoids: smooth, deterministic displacement."""
    out = np.zeros(p.shape[0])
    amp = 1.0
    for _ in range(octaves):
        k = rng.normal(size=(3, 3)) * 2.0
        ph = rng.uniform(0, 2 * math.pi, size=3)
        out += amp * np.sin(p @ k + ph).sum(axis=1) / 3.0
        amp *= 0.5
    return out


def _dome_texture(width, height, seed, hotspots=3, sigma=2.0) -> np.ndarray:
    """Lat-long RGBA32F dome: log-normal luminance (`sigma`) + `hotspots` Gaussian hotspots."""
    rng = np.random.default_rng(seed)
    # Smooth log-normal field: low-resolution Gaussian noise upsampled.
    lw, lh = 64, 32
    g = rng.normal(size=(lh, lw))
    ys = np.linspace(0, lh - 1, height)
    xs = np.linspace(0, lw - 1, width)
    y0 = np.floor(ys).astype(int)
    x0 = np.floor(xs).astype(int)
    y1 = np.minimum(y0 + 1, lh - 1)
    x1 = (x0 + 1) % lw
    fy = (ys - y0)[:, None]
    fx = (xs - x0)[None, :]
    field = (g[y0][:, x0] * (1 - fx) * (1 - fy) + g[y0][:, x1] * fx * (1 - fy) +
             g[y1][:, x0] * (1 - fx) * fy + g[y1][:, x1] * fx * fy)
    field = field / max(field.std(), 1e-6)
    lum = np.exp(sigma * field - sigma)  # log-normal
    v = (np.arange(height) + 0.5) / height
    u = (np.arange(width) + 0.5) / width
    uu, vv = np.meshgrid(u, v)
    for _ in range(hotspots):
        cu, cv = rng.uniform(0.0, 1.0), rng.uniform(0.55, 0.9)
        s = rng.uniform(0.01, 0.03)
        du = np.minimum(np.abs(uu - cu), 1.0 - np.abs(uu - cu))
        lum += rng.uniform(200.0, 800.0) * np.exp(-(du ** 2 + (vv - cv) ** 2) / (2 * s * s))
    tint = rng.uniform(0.7, 1.0, size=3)
    rgba = np.empty((height, width, 4), np.float32)
    for c in range(3):
        rgba[..., c] = lum * tint[c]
    rgba[..., 3] = 1.0
    return rgba


def heavy_geometry(width=1920, height=1080, spp=64, max_bounces=8, seed=0, sphere_level=3,
                   grid_vertices=581, dome_size=(2048, 1024), instanced=False) -> Workload:
    """The 1.0M-triangle scene: a noise-displaced heightfield and 256 displaced
    icospheres, lit by a lat-long HDR dome. With instanced=True the spheres are
    instances (hdcx_instancer_desc) of four displaced icosphere prototypes,
    each with its own uniform scale, rotation about y and position: the same
    triangle count and layout, given as instancers instead of flattened
    copies."""
    if instanced:
        return _heavy_instanced(width, height, spp, max_bounces, seed, sphere_level, grid_vertices, dome_size)
    rng = np.random.default_rng(seed)
    s = Scene(revision=1)
    # Material palette: Lambert, GGX dielectric (reflective over diffuse), GGX conductor.
    mats = []
    for i in range(8):
        mats.append(Material(id=f"/lambert{i}", base_color=rng.uniform(0.1, 0.9, 3).tolist(),
                             specular_weight=0.0))
    for i in range(16):
        mats.append(Material(id=f"/dielectric{i}", base_color=rng.uniform(0.05, 0.8, 3).tolist(),
                             roughness=float(rng.uniform(0.05, 0.8)), index_of_refraction=1.5,
                             specular_weight=1.0))
        mats[-1].roughness_v = mats[-1].roughness
    for i in range(8):
        m = Material(id=f"/conductor{i}", base_color=rng.uniform(0.5, 1.0, 3).tolist(), metalness=1.0,
                     roughness=float(rng.uniform(0.05, 0.6)))
        m.roughness_v = m.roughness
        mats.append(m)
    s.materials = mats
    families = [[m.id for m in mats[:8]], [m.id for m in mats[8:24]], [m.id for m in mats[24:]]]

    def pick_ids(n):
        fam = rng.integers(0, 3, size=n)
        idx = np.array([rng.integers(0, len(families[f])) for f in fam])
        return [families[f][i] for f, i in zip(fam, idx)]

    # Heightfield.
    n = grid_vertices
    xs = np.linspace(-12.0, 12.0, n)
    X, Z = np.meshgrid(xs, xs)
    pts = np.stack([X.ravel(), np.zeros(n * n), Z.ravel()], axis=1)
    H = 0.6 * _noise3(pts * 0.35, rng, 5)
    pts[:, 1] = H
    ii, jj = np.meshgrid(np.arange(n - 1), np.arange(n - 1), indexing="ij")
    a = (ii * n + jj).ravel()
    b = a + 1
    c = a + n
    d = c + 1
    tris = np.stack([np.stack([a, c, b], 1), np.stack([b, c, d], 1)], 1).reshape(-1, 3).astype(np.uint32)
    s.meshes.append(Mesh(id="/ground", positions=pts.astype(np.float32).ravel(), indices=tris.ravel(),
                         material_id="/lambert0", triangle_material_ids=pick_ids(len(tris))))
    # Instanced displaced icospheres, flattened.
    base_v, base_f = _icosphere(sphere_level)
    all_v, all_f = [], []
    offset = 0
    for k in range(256):
        gx, gz = k % 16, k // 16
        cx = -10.5 + gx * 1.4 + rng.uniform(-0.3, 0.3)
        cz = -10.5 + gz * 1.4 + rng.uniform(-0.3, 0.3)
        r = rng.uniform(0.25, 0.55)
        disp = 1.0 + 0.18 * _noise3(base_v * 2.0, rng, 3)
        v = base_v * (r * disp)[:, None]
        v = v + np.array([cx, 1.2 + r, cz])
        all_v.append(v)
        all_f.append(base_f + offset)
        offset += len(v)
    sv = np.concatenate(all_v).astype(np.float32)
    sf = np.concatenate(all_f).astype(np.uint32)
    s.meshes.append(Mesh(id="/spheres", positions=sv.ravel(), indices=sf.ravel(), material_id="/lambert0",
                         triangle_material_ids=pick_ids(len(sf))))
    dw, dh = dome_size
    dome = _dome_texture(dw, dh, seed + 7)
    s.textures.append(Texture(id="dome#hdr", width=dw, height=dh, rgba_float=dome.ravel()))
    s.lights.append(Light(id="/dome", type=DOME, intensity=1.0, texture="dome#hdr", texture_format=LATLONG))
    cam = look_at_camera((0.0, 7.5, 17.0), (0.0, 0.0, -1.0), (0.0, 1.0, 0.0), 45.0, width / height)
    return Workload("heavy-geometry-1.0M-tri-dome", s, cam, width, height, spp, max_bounces)


def _heavy_instanced(width, height, spp, max_bounces, seed, sphere_level, grid_vertices, dome_size) -> Workload:
    from .scene import Instancer
    flat = heavy_geometry(width, height, spp, max_bounces, seed, sphere_level, grid_vertices, dome_size)
    s = flat.scene
    s.meshes = [m for m in s.meshes if m.id != "/spheres"]
    rng = np.random.default_rng(seed + 101)
    ids = [m.id for m in s.materials]
    base_v, base_f = _icosphere(sphere_level)
    protos = 4
    for k in range(protos):
        disp = 1.0 + 0.18 * _noise3(base_v * 2.0, rng, 3)
        v = (base_v * disp[:, None]).astype(np.float32)
        tri_ids = [ids[int(i)] for i in rng.integers(0, len(ids), size=len(base_f))]
        s.meshes.append(Mesh(id=f"/sphere{k}", positions=v.ravel(), indices=base_f.astype(np.uint32).ravel(),
                             material_id="/lambert0", triangle_material_ids=tri_ids))
    transforms = [[] for _ in range(protos)]
    for k in range(256):
        gx, gz = k % 16, k // 16
        cx = -10.5 + gx * 1.4 + rng.uniform(-0.3, 0.3)
        cz = -10.5 + gz * 1.4 + rng.uniform(-0.3, 0.3)
        r = rng.uniform(0.25, 0.55)
        th = rng.uniform(0.0, 2.0 * np.pi)
        c, sn = np.cos(th), np.sin(th)
        M = np.array([[r * c, 0.0, -r * sn, 0.0], [0.0, r, 0.0, 0.0], [r * sn, 0.0, r * c, 0.0],
                      [cx, 1.2 + r, cz, 1.0]], dtype=np.float64)
        transforms[k % protos].append(M)
    s.instancers = [Instancer(f"/sphere{k}", np.array(transforms[k])) for k in range(protos)]
    return Workload("heavy-geometry-1.0M-tri-instanced", s, flat.camera, width, height, spp, max_bounces)


def _torus(major: float, minor: float, segments: int, rings: int):
    u = np.arange(segments) * (2 * math.pi / segments)
    v = np.arange(rings) * (2 * math.pi / rings)
    U, V = np.meshgrid(u, v, indexing="ij")
    x = (major + minor * np.cos(V)) * np.cos(U)
    z = (major + minor * np.cos(V)) * np.sin(U)
    y = minor * np.sin(V)
    verts = np.stack([x.ravel(), y.ravel(), z.ravel()], 1)
    i, j = np.meshgrid(np.arange(segments), np.arange(rings), indexing="ij")
    a = (i * rings + j).ravel()
    b = (((i + 1) % segments) * rings + j).ravel()
    c = (i * rings + (j + 1) % rings).ravel()
    d = (((i + 1) % segments) * rings + (j + 1) % rings).ravel()
    faces = np.stack([np.stack([a, c, b], 1), np.stack([b, c, d], 1)], 1).reshape(-1, 3)
    return verts, faces.astype(np.uint32)


def _grid_top(x0, x1, z0, z1, y, nx, nz):
    xs = np.linspace(x0, x1, nx + 1)
    zs = np.linspace(z0, z1, nz + 1)
    X, Z = np.meshgrid(xs, zs, indexing="ij")
    verts = np.stack([X.ravel(), np.full(X.size, y), Z.ravel()], 1)
    i, j = np.meshgrid(np.arange(nx), np.arange(nz), indexing="ij")
    a = (i * (nz + 1) + j).ravel()
    b = a + (nz + 1)
    c = a + 1
    d = b + 1
    faces = np.stack([np.stack([a, c, b], 1), np.stack([b, c, d], 1)], 1).reshape(-1, 3)
    return verts, faces.astype(np.uint32)


def spectral_stress(width=1280, height=720, spp=256, max_bounces=8, seed=0, sphere_level=6,
                    torus_segments=(256, 192), leaf_count=2048, mask_size=64,
                    dome_size=(1024, 512)) -> Workload:
    """~200k triangles: a dispersive, absorbing, scattering glass sphere (g = 0.7),
    two small glass spheres (g = -0.3 and 0), a subsurface torus (radius
    (1, 0.2, 0.1)) and opacity-cutout leaves (seeded fp32 mask, 25% of texels
    cut) on a plinth, under a lat-long dome and a rect light. Every dielectric
    has transmission 1, dispersion scale 1, an Abbe number drawn from
    U{20..60} and transmission depth 0.5; the leaves make the scene
    non-opaque, so every ray takes the opacity any-hit path."""
    rng = np.random.default_rng(seed)
    s = Scene(revision=1)
    mats = [Material(id="/plinth", base_color=[0.55, 0.52, 0.48], roughness=0.45, specular_weight=0.5)]
    for name, g, color in (("/glass_forward", 0.7, [0.85, 0.6, 0.4]), ("/glass_back", -0.3, [0.5, 0.7, 0.9]),
                           ("/glass_iso", 0.0, [0.7, 0.9, 0.6])):
        m = Material(id=name, base_color=[1.0, 1.0, 1.0], transmission=1.0, transmission_color=color,
                     transmission_depth=0.5, transmission_scatter=[0.6, 0.6, 0.6],
                     transmission_scatter_anisotropy=g, transmission_dispersion_scale=1.0,
                     transmission_dispersion_abbe_number=float(rng.integers(20, 61)), index_of_refraction=1.5,
                     roughness=0.0, specular_weight=1.0)
        m.roughness_v = 0.0
        mats.append(m)
    mats.append(Material(id="/subsurface", base_color=[0.9, 0.62, 0.5], subsurface=1.0,
                         subsurface_color=[0.9, 0.62, 0.5], subsurface_radius=[1.0, 0.2, 0.1],
                         subsurface_scale=0.25, roughness=0.35, specular_weight=0.5))
    mats.append(Material(id="/leaf", base_color=[0.2, 0.55, 0.12], specular_weight=0.25, roughness=0.6,
                         opacity_texture="leafmask#raw"))
    s.materials = mats

    # Plinth: subdivided top (64 x 48) and four sides.
    tv, tf = _grid_top(-4.0, 4.0, -3.0, 3.0, 0.0, 64, 48)
    side_v, side_f = [], []
    for quad in (((-4, -0.5, 3), (4, -0.5, 3), (4, 0, 3), (-4, 0, 3)),
                 ((4, -0.5, -3), (-4, -0.5, -3), (-4, 0, -3), (4, 0, -3)),
                 ((4, -0.5, 3), (4, -0.5, -3), (4, 0, -3), (4, 0, 3)),
                 ((-4, -0.5, -3), (-4, -0.5, 3), (-4, 0, 3), (-4, 0, -3))):
        base = len(tv) + len(side_v)
        side_v += [list(map(float, p)) for p in quad]
        side_f += [[base, base + 1, base + 2], [base, base + 2, base + 3]]
    pv = np.concatenate([tv, np.asarray(side_v)])
    pf = np.concatenate([tf, np.asarray(side_f, np.uint32)])
    s.meshes.append(Mesh(id="/plinth", positions=pv.astype(np.float32).ravel(), indices=pf.ravel(),
                         material_id="/plinth"))

    # Glass spheres.
    sv, sf = _icosphere(sphere_level)
    s.meshes.append(Mesh(id="/sphere", positions=(sv * 1.0 + np.array([-1.7, 1.0, 0.2])).astype(np.float32).ravel(),
                         indices=sf.ravel(), material_id="/glass_forward"))
    small_v, small_f = _icosphere(max(sphere_level - 2, 1))
    for k, (mat, centre) in enumerate((("/glass_back", (0.2, 0.45, 1.6)), ("/glass_iso", (-0.4, 0.45, -1.7)))):
        s.meshes.append(Mesh(id=f"/small{k}",
                             positions=(small_v * 0.45 + np.array(centre)).astype(np.float32).ravel(),
                             indices=small_f.ravel(), material_id=mat))

    # Subsurface torus, tilted.
    ov, of = _torus(1.0, 0.38, *torus_segments)
    tilt = math.radians(25.0)
    rot = np.array([[1, 0, 0], [0, math.cos(tilt), -math.sin(tilt)], [0, math.sin(tilt), math.cos(tilt)]])
    ov = ov @ rot.T + np.array([1.7, 0.85, 0.0])
    s.meshes.append(Mesh(id="/torus", positions=ov.astype(np.float32).ravel(), indices=of.ravel(),
                         material_id="/subsurface"))

    # Leaves: random quads in a bush behind the objects, UV 0..1 per quad.
    lv, lf, luv = [], [], []
    for k in range(leaf_count):
        c = np.array([rng.uniform(-3.5, 3.5), rng.uniform(0.4, 3.2), rng.uniform(-2.9, -1.6)])
        n = rng.normal(size=3)
        n /= np.linalg.norm(n)
        t = np.cross(n, [0.0, 1.0, 0.0] if abs(n[1]) < 0.9 else [1.0, 0.0, 0.0])
        t /= np.linalg.norm(t)
        b = np.cross(n, t)
        size = rng.uniform(0.12, 0.3)
        corners = [c - size * t - size * b, c + size * t - size * b, c + size * t + size * b, c - size * t + size * b]
        base = 4 * k
        lv += corners
        lf += [[base, base + 1, base + 2], [base, base + 2, base + 3]]
        luv += [0.0, 0.0, 1.0, 0.0, 1.0, 1.0, 0.0, 0.0, 1.0, 1.0, 0.0, 1.0]
    s.meshes.append(Mesh(id="/leaves", positions=np.asarray(lv, np.float32).ravel(),
                         indices=np.asarray(lf, np.uint32).ravel(), texcoords=luv, material_id="/leaf"))
    mask = (rng.random((mask_size, mask_size)) >= 0.25).astype(np.float32)
    rgba = np.repeat(mask[..., None], 4, axis=2)
    rgba[..., 3] = 1.0
    s.textures.append(Texture(id="leafmask#raw", source_path="synthetic", width=mask_size, height=mask_size,
                              srgb=False, rgba_float=rgba.ravel()))

    dw, dh = dome_size
    # Lighting: a sky dome only, log-normal (sigma 0.5) without sun-like
    # hotspots. A hotspot seen through the delta glass can only be found by
    # BSDF sampling, and a small area light sampled into the glass's
    # near-delta reflection lobe (the integrator applies no MIS to analytic
    # lights) makes fireflies that keep even a 4096-spp render above 20%
    # relative RMSE; the dome is sampled with MIS.
    dome = _dome_texture(dw, dh, seed + 11, hotspots=0, sigma=0.5)
    s.textures.append(Texture(id="stressdome#hdr", width=dw, height=dh, rgba_float=dome.ravel()))
    s.lights.append(Light(id="/dome", type=DOME, intensity=1.0, texture="stressdome#hdr", texture_format=LATLONG))
    cam = look_at_camera((0.0, 3.0, 7.8), (0.0, 0.9, 0.0), (0.0, 1.0, 0.0), 40.0, width / height)
    return Workload("spectral-stress-200k-tri", s, cam, width, height, spp, max_bounces)


BATCH_RESOLUTIONS = ((256, 256), (512, 512), (1280, 720), (1920, 1080))


def _c2_palette(rng, prefix=""):
    """The heavy-geometry material families: Lambert, GGX dielectric over
    diffuse, GGX conductor."""
    mats = []
    for i in range(4):
        mats.append(Material(id=f"{prefix}/lambert{i}", base_color=rng.uniform(0.1, 0.9, 3).tolist(),
                             specular_weight=0.0))
    for i in range(4):
        m = Material(id=f"{prefix}/dielectric{i}", base_color=rng.uniform(0.05, 0.8, 3).tolist(),
                     roughness=float(rng.uniform(0.05, 0.8)), index_of_refraction=1.5, specular_weight=1.0)
        m.roughness_v = m.roughness
        mats.append(m)
    for i in range(4):
        m = Material(id=f"{prefix}/conductor{i}", base_color=rng.uniform(0.5, 1.0, 3).tolist(), metalness=1.0,
                     roughness=float(rng.uniform(0.05, 0.6)))
        m.roughness_v = m.roughness
        mats.append(m)
    return mats


def batch_job(index: int, seed: int = 0, dome_size=(1024, 512)) -> Workload:
    """Job `index` of the multi-job batch: triangles log-uniform in [10k, 2M]
    (a heightfield carrying ~70% of them plus displaced level-3 icospheres),
    resolution drawn from BATCH_RESOLUTIONS, spp uniform in {4..128},
    per-triangle materials of the heavy-geometry families, one lat-long dome
    and 1-8 rect/disk/sphere lights. A pure function of (index, seed)."""
    from .scene import DISK, SPHERE
    rng = np.random.default_rng([seed, index])
    target = int(round(math.exp(rng.uniform(math.log(10_000), math.log(2_000_000)))))
    width, height = BATCH_RESOLUTIONS[int(rng.integers(0, len(BATCH_RESOLUTIONS)))]
    spp = int(rng.integers(4, 129))
    s = Scene(revision=1)
    s.materials = _c2_palette(rng)
    ids = [m.id for m in s.materials]
    n = max(8, int(round(math.sqrt(0.7 * target / 2.0))) + 1)
    half = 10.0
    xs = np.linspace(-half, half, n)
    X, Z = np.meshgrid(xs, xs)
    pts = np.stack([X.ravel(), np.zeros(n * n), Z.ravel()], axis=1)
    pts[:, 1] = 0.6 * _noise3(pts * 0.35, rng, 4)
    ii, jj = np.meshgrid(np.arange(n - 1), np.arange(n - 1), indexing="ij")
    a = (ii * n + jj).ravel()
    tris = np.stack([np.stack([a, a + n, a + 1], 1), np.stack([a + 1, a + n, a + n + 1], 1)], 1)
    tris = tris.reshape(-1, 3).astype(np.uint32)
    pick = rng.integers(0, len(ids), size=len(tris))
    s.meshes.append(Mesh(id="/ground", positions=pts.astype(np.float32).ravel(), indices=tris.ravel(),
                         material_id=ids[0], triangle_material_ids=[ids[k] for k in pick]))
    spheres = max(0, int(round((target - len(tris)) / 1280.0)))
    if spheres:
        base_v, base_f = _icosphere(3)
        all_v, all_f = [], []
        for k in range(spheres):
            r = rng.uniform(0.2, 0.5)
            c = np.array([rng.uniform(-half + 1, half - 1), 1.0 + r, rng.uniform(-half + 1, half - 1)])
            disp = 1.0 + 0.15 * np.sin(base_v @ rng.normal(size=(3,)) * 3.0 + rng.uniform(0, 6.28))
            all_v.append(base_v * (r * disp)[:, None] + c)
            all_f.append(base_f + k * len(base_v))
        sf = np.concatenate(all_f).astype(np.uint32)
        pick = rng.integers(0, len(ids), size=len(sf))
        s.meshes.append(Mesh(id="/spheres", positions=np.concatenate(all_v).astype(np.float32).ravel(),
                             indices=sf.ravel(), material_id=ids[0], triangle_material_ids=[ids[k] for k in pick]))
    dw, dh = dome_size
    s.textures.append(Texture(id="dome#hdr", width=dw, height=dh, rgba_float=_dome_texture(dw, dh, seed + 1000 + index).ravel()))
    s.lights.append(Light(id="/dome", type=DOME, intensity=1.0, texture="dome#hdr", texture_format=LATLONG))
    for k in range(int(rng.integers(1, 9))):
        kind = (RECT, DISK, SPHERE)[int(rng.integers(0, 3))]
        pos = [float(rng.uniform(-6, 6)), float(rng.uniform(3, 7)), float(rng.uniform(-6, 6))]
        color = rng.uniform(0.6, 1.0, 3).tolist()
        size = float(rng.uniform(0.3, 1.2))
        if kind == SPHERE:
            light = Light(id=f"/light{k}", type=SPHERE, color=color, intensity=float(rng.uniform(5, 30)),
                          position=pos, radius=size * 0.5)
        else:
            light = Light(id=f"/light{k}", type=kind, color=color, intensity=float(rng.uniform(5, 30)),
                          position=pos, basis_x=[1.0, 0.0, 0.0], basis_y=[0.0, 0.0, 1.0], basis_z=[0.0, 1.0, 0.0],
                          axis_u=[size, 0.0, 0.0], axis_v=[0.0, 0.0, size], width=size, height=size,
                          radius=size * 0.5, area=size * size if kind == RECT else math.pi * (size * 0.5) ** 2)
        s.lights.append(light)
    eye = (float(rng.uniform(-4, 4)), float(rng.uniform(5, 8)), float(rng.uniform(12, 16)))
    cam = look_at_camera(eye, (0.0, 0.5, 0.0), (0.0, 1.0, 0.0), 45.0, width / height)
    return Workload(f"batch-job-{index}", s, cam, width, height, spp, 8)


def batch_jobs(count: int = 64, seed: int = 0, **kw):
    """The multi-job batch: `count` jobs of batch_job."""
    return [batch_job(i, seed, **kw) for i in range(count)]


def triangle_count(scene: Scene) -> int:
    return sum(len(m.indices) // 3 for m in scene.meshes)
