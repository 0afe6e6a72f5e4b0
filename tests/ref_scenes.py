"""Scenes of the reference's GPU integration test, restated as Scene objects.

The base scene, camera and every variant follow tests/path_tracer_tests.cpp of
hdCodex (line numbers cited per variant): a triangle at z = -3 seen by a 64x64
camera, a green sRGB base-color texture, a blue dome and a textured rect light.
"""
from __future__ import annotations

from hdcodex_b200.scene import (CYLINDER, DISK, DISTANT, DOME, RECT, SPHERE, Light, Material,
                                Mesh, Scene, Texture, camera)

WIDTH = 64
HEIGHT = 64
CENTER = (HEIGHT // 2, WIDTH // 2)
CORNER = (0, 0)


def base_camera():
    # path_tracer_tests.cpp:132-137
    return camera((0.0, 0.0, 0.0), (-1.0, -1.0, -1.0), (2.0, 0.0, 0.0), (0.0, 2.0, 0.0))


def z_up_camera():
    # path_tracer_tests.cpp:478-483
    return camera((0.0, 0.0, 0.0), (-1.0, -1.0, -1.0), (2.0, 0.0, 0.0), (0.0, 0.0, 2.0))


def base_scene() -> Scene:
    # path_tracer_tests.cpp:36-129
    s = Scene(revision=1)
    s.meshes.append(Mesh(
        id="/triangle",
        positions=[-1.25, -1.0, -3.0, 1.25, -1.0, -3.0, 0.0, 1.2, -3.0],
        indices=[0, 1, 2],
        texcoords=[0.0, 0.0, 1.0, 0.0, 0.5, 1.0],
        material_id="/red",
    ))
    s.materials.append(Material(id="/red", base_color=[1.0, 1.0, 1.0], metalness=0.15,
                                roughness=0.3, base_color_texture="green#srgb"))
    s.textures += [
        Texture(id="green#srgb", source_path="synthetic", width=1, height=1, srgb=True,
                rgba=[16, 220, 32, 255]),
        Texture(id="scatter#raw", source_path="synthetic", width=1, height=1, srgb=False,
                rgba=[255, 255, 255, 255]),
        Texture(id="synthetic-udim#srgb#udim=1001", source_path="synthetic.1001",
                udim_set_id="synthetic-udim#srgb", udim_tile=1001, width=1, height=1, srgb=True,
                rgba=[230, 16, 16, 255]),
        Texture(id="synthetic-udim#srgb#udim=1002", source_path="synthetic.1002",
                udim_set_id="synthetic-udim#srgb", udim_tile=1002, width=1, height=1, srgb=True,
                rgba=[16, 24, 230, 255]),
        Texture(id="rect#hdr", source_path="synthetic", width=1, height=1, srgb=False,
                rgba_float=[2.0, 2.0, 2.0, 1.0]),
        Texture(id="spectral-gradient#hdr", source_path="synthetic", width=4, height=1, srgb=False,
                rgba_float=[3.0, 0.02, 0.02, 1.0, 0.02, 3.0, 0.02, 1.0,
                            0.02, 0.02, 3.0, 1.0, 3.0, 3.0, 3.0, 1.0]),
    ]
    s.lights += [
        Light(id="/dome", type=DOME, color=[0.08, 0.16, 0.8], intensity=0.35),
        Light(id="/rect", type=RECT, color=[1.0, 0.92, 0.82], intensity=50.0, texture="rect#hdr",
              basis_x=[0.817, -0.576, 0.0], basis_y=[0.184, 0.261, -0.947],
              basis_z=[0.547, 0.775, 0.319], position=[3.282, 4.650, -1.086],
              axis_u=[1.634, -1.152, 0.0], axis_v=[0.368, 0.522, -1.894], width=2.0, height=2.0,
              area=4.0),
    ]
    return s


def analytic_lights():
    # path_tracer_tests.cpp:169-203
    return [
        Light(id="/disk", type=DISK, intensity=20.0, position=[0.0, 0.0, -1.5],
              axis_u=[0.75, 0.0, 0.0], axis_v=[0.0, 0.75, 0.0], area=1.7671459),
        Light(id="/sphere", type=SPHERE, intensity=20.0, position=[0.0, 0.0, -1.5], radius=0.35,
              area=1.5393804),
        Light(id="/cylinder", type=CYLINDER, intensity=20.0, position=[0.0, 0.0, -1.5],
              axis_u=[1.0, 0.0, 0.0], radius=0.25, length=1.0, area=1.5707963),
        Light(id="/distant", type=DISTANT, intensity=1.0, angle=0.53),
    ]


def selection_scene() -> Scene:
    # path_tracer_tests.cpp:217-226: 63 black domes and the rect light.
    s = base_scene()
    rect = s.lights[1]
    s.lights = [Light(id=f"/black{i}", type=DOME, intensity=0.0) for i in range(63)] + [rect]
    return s


def mesh_light_scene(emission_weight=1.0) -> Scene:
    # path_tracer_tests.cpp:237-283
    s = Scene(revision=2)
    s.meshes = [
        Mesh(id="/receiver", positions=[-1.25, -1.0, -3.0, 1.25, -1.0, -3.0, 0.0, 1.2, -3.0],
             indices=[0, 1, 2], material_id="/receiverMaterial"),
        Mesh(id="/emitter", positions=[0.35, 0.35, -1.8, 1.10, 0.35, -1.8, 0.70, 1.00, -1.8],
             indices=[0, 1, 2], material_id="/emitterMaterial"),
    ]
    s.materials = [
        Material(id="/receiverMaterial", base_color=[0.8, 0.8, 0.8], roughness=0.6),
        Material(id="/emitterMaterial", base_color=[0.0, 0.0, 0.0], emission=[16.0, 12.0, 8.0],
                 emission_weight=emission_weight),
    ]
    s.lights = [Light(id="/blackDome", type=DOME, intensity=0.0)]
    return s


def variant(name: str) -> Scene:
    """Named variants of the base scene from path_tracer_tests.cpp."""
    s = base_scene()
    m = s.materials[0]
    if name == "base":
        pass
    elif name == "oren_nayar":  # :294-298
        m.diffuse_model = 1
        m.diffuse_roughness = 0.85
    elif name == "udim":  # :313-318
        s.meshes[0].texcoords = [1.1, 0.1, 1.9, 0.1, 1.5, 0.9]
        m.base_color_texture = "synthetic-udim#srgb"
    elif name == "authored_normals":  # :334-341
        s.meshes[0].normals = [0.6, 0.85, 0.35] * 3
    elif name in ("glossy", "matte_black", "coated"):  # :345-371
        s.meshes[0].normals = [0.3446, 0.4881, 0.8027] * 3
        m.base_color = [0.0, 0.0, 0.0]
        m.base_color_texture = ""
        m.roughness = 0.08
        m.specular_weight = 1.0 if name != "matte_black" else 0.0
        if name == "coated":
            m.specular_weight = 0.0
            m.coat = 1.0
            m.coat_roughness = 0.08
    elif name == "subsurface":  # :380-384
        m.subsurface_color = [0.02, 0.05, 1.0]
        m.subsurface_scale = 0.0
        m.subsurface_texture = "scatter#raw"
    elif name == "cutout":  # :391-393
        m.opacity = 0.0
    elif name in ("opaque_black", "translucent"):  # :398-414
        m.base_color = [0.0, 0.0, 0.0]
        m.base_color_texture = ""
        m.diffuse_weight = 0.0
        m.specular_weight = 0.0
        m.coat = 0.0
        if name == "translucent":
            m.translucent_weight = 1.0
            m.translucent_color = [1.0, 0.02, 0.01]
    elif name in ("thin_walled", "nondispersive", "dispersive"):  # :416-449
        m.base_color = [0.0, 0.0, 0.0]
        m.base_color_texture = ""
        m.diffuse_weight = 1.0
        m.specular_weight = 0.0
        m.transmission = 1.0
        m.metalness = 0.0
        if name == "thin_walled":
            m.transmission_color = [1.0, 0.05, 0.02]
            m.thin_walled = True
        else:
            m.transmission_color = [1.0, 1.0, 1.0]
            s.lights = s.lights[:1]
            s.lights[0].color = [1.0, 1.0, 1.0]
            s.lights[0].intensity = 1.0
            s.lights[0].texture = "spectral-gradient#hdr"
            if name == "dispersive":
                m.transmission_dispersion_scale = 1.0
                m.transmission_dispersion_abbe_number = 9.0
    elif name in ("fallback", "fallback_zup"):  # :451-490
        s.lights = []
        s.meshes[0].material_id = ""
        s.meshes[0].display_color = [0.05, 0.8, 0.1]
        m.base_color = [0.8, 0.8, 0.8]
        m.base_color_texture = ""
        m.roughness = 1.0
        if name == "fallback_zup":
            s.meshes[0].positions = [-1.25, -3.0, -1.0, 0.0, -3.0, 1.2, 1.25, -3.0, -1.0]
    else:
        raise KeyError(name)
    return s


def fuzz_material(rng, material_id: str) -> Material:
    """A seeded random material over the closure ABI: every diffuse model,
    anisotropic GGX, coat, sheen (both modes), translucency, subsurface,
    transmission (dispersive, scattering, thin-walled) and emission; opacity 1
    (cut-outs agree with the reference only in expectation)."""
    m = Material(id=material_id)
    m.base_color = rng.uniform(0.02, 0.95, 3).tolist()
    m.diffuse_model = int(rng.integers(0, 4))
    m.diffuse_roughness = float(rng.uniform(0, 1))
    m.diffuse_weight = float(rng.choice([1.0, rng.uniform(0, 1)]))
    m.metalness = float(rng.choice([0.0, rng.uniform(0, 1), 1.0]))
    m.roughness = float(rng.uniform(0.02, 1))
    m.roughness_v = float(rng.choice([m.roughness, rng.uniform(0.02, 1)]))
    m.specular_weight = float(rng.choice([0.0, 1.0, rng.uniform(0, 1)]))
    m.specular_color = rng.uniform(0.3, 1, 3).tolist()
    m.index_of_refraction = float(rng.uniform(1.1, 2.2))
    if rng.random() < 0.4:
        m.coat = float(rng.uniform(0, 1))
        m.coat_roughness = float(rng.uniform(0.01, 0.6))
        m.coat_roughness_v = float(rng.choice([m.coat_roughness, rng.uniform(0.01, 0.6)]))
        m.coat_color = rng.uniform(0.5, 1, 3).tolist()
        m.coat_index_of_refraction = float(rng.uniform(1.2, 2.0))
    if rng.random() < 0.4:
        m.sheen = float(rng.uniform(0, 1))
        m.sheen_roughness = float(rng.uniform(0.05, 1))
        m.sheen_mode = int(rng.integers(0, 2))
        m.sheen_color = rng.uniform(0.2, 1, 3).tolist()
    if rng.random() < 0.3:
        m.translucent_weight = float(rng.uniform(0, 1))
        m.translucent_color = rng.uniform(0.1, 1, 3).tolist()
    if rng.random() < 0.3:
        m.subsurface = float(rng.uniform(0, 1))
        m.subsurface_color = rng.uniform(0.1, 0.99, 3).tolist()
        m.subsurface_radius = rng.uniform(0.01, 0.5, 3).tolist()
        m.subsurface_scale = float(rng.uniform(0.05, 1))
        m.subsurface_scatter_anisotropy = float(rng.uniform(-0.8, 0.8))
    if rng.random() < 0.3:
        m.transmission = float(rng.uniform(0.3, 1))
        m.transmission_color = rng.uniform(0.3, 1, 3).tolist()
        m.transmission_depth = float(rng.choice([0.0, rng.uniform(0.05, 1)]))
        m.transmission_scatter = (rng.uniform(0, 2, 3) if rng.random() < 0.5 else [0.0, 0.0, 0.0])
        m.transmission_scatter = [float(x) for x in m.transmission_scatter]
        m.transmission_scatter_anisotropy = float(rng.uniform(-0.8, 0.8))
        if rng.random() < 0.5:
            m.transmission_dispersion_scale = float(rng.uniform(0.2, 1))
            m.transmission_dispersion_abbe_number = float(rng.uniform(9, 60))
        m.thin_walled = bool(rng.random() < 0.3)
    if rng.random() < 0.15:
        m.emission = rng.uniform(0.5, 5, 3).tolist()
        m.emission_weight = float(rng.uniform(0.2, 1))
    return m


def fuzz_box(seed: int, size: int = 40):
    """The closed box (5 walls, 2 boxes, a rect light) with seeded random
    materials on walls and boxes, and at random a dome and a sphere light."""
    import numpy as np

    from hdcodex_b200 import workloads
    rng = np.random.default_rng(seed)
    wl = workloads.closed_box(width=size, height=size, spp=4)
    s = wl.scene
    s.materials = [fuzz_material(rng, i) for i in ("/white", "/red", "/green", "/tallBox", "/shortBox")]
    for mesh in s.meshes:
        if mesh.id == "/tall":
            mesh.material_id = "/tallBox"
        elif mesh.id == "/short":
            mesh.material_id = "/shortBox"
    if rng.random() < 0.5:
        s.lights.append(Light(id="/dome", type=DOME, color=rng.uniform(0.1, 1, 3).tolist(),
                              intensity=float(rng.uniform(0.1, 1))))
    if rng.random() < 0.4:
        s.lights.append(Light(id="/sphere", type=SPHERE, intensity=float(rng.uniform(1, 10)),
                              position=[0.5, 0.7, 0.6], radius=0.05, area=0.0314159))
    return wl


def _fuzz_frame(rng):
    import numpy as np
    z = rng.normal(size=3)
    z /= np.linalg.norm(z)
    a = np.array([1.0, 0.0, 0.0]) if abs(z[0]) < 0.9 else np.array([0.0, 1.0, 0.0])
    x = np.cross(a, z)
    x /= np.linalg.norm(x)
    return x, np.cross(z, x), z


def fuzz_light(rng, light_id: str, textures) -> Light:
    """A seeded random light of any type: placement and frame, colour,
    temperature tint, exposure, diffuse/specular factors, normalisation,
    visibility, shaping cone and focus, shadow controls, and (rect and dome)
    a texture from `textures`."""
    kind = int(rng.choice([RECT, DISK, SPHERE, CYLINDER, DISTANT, DOME]))
    x, y, z = _fuzz_frame(rng)
    l = Light(id=light_id, type=kind)
    l.color = rng.uniform(0.2, 1, 3).tolist()
    l.temperature_color = rng.uniform(0.6, 1, 3).tolist()
    l.intensity = float(rng.uniform(0.5, 8))
    l.exposure = float(rng.uniform(-1, 1))
    l.diffuse = float(rng.choice([1.0, rng.uniform(0, 1)]))
    l.specular = float(rng.choice([1.0, rng.uniform(0, 1)]))
    l.normalize = bool(rng.random() < 0.5)
    l.visible = bool(rng.random() < 0.7)
    l.basis_x, l.basis_y, l.basis_z = x.tolist(), y.tolist(), z.tolist()
    l.position = rng.uniform(0.15, 0.85, 3).tolist()
    l.width, l.height = float(rng.uniform(0.05, 0.4)), float(rng.uniform(0.05, 0.4))
    l.axis_u = (x * l.width / 2).tolist()
    l.axis_v = (y * l.height / 2).tolist()
    l.radius = float(rng.uniform(0.02, 0.15))
    l.length = float(rng.uniform(0.05, 0.4))
    l.angle = float(rng.uniform(0.2, 8.0))
    l.area = float(rng.uniform(0.01, 0.2))
    if rng.random() < 0.5:
        l.shaping_focus = float(rng.uniform(0, 2))
        l.shaping_focus_tint = rng.uniform(0, 1, 3).tolist()
        l.shaping_cone_angle = float(rng.uniform(20, 180))
        l.shaping_cone_softness = float(rng.uniform(0, 1))
    l.shadow_enable = bool(rng.random() < 0.85)
    if rng.random() < 0.4:
        l.shadow_color = rng.uniform(0, 0.5, 3).tolist()
        l.shadow_distance = float(rng.choice([-1.0, rng.uniform(0.1, 1.5)]))
        l.shadow_falloff = float(rng.choice([-1.0, rng.uniform(0.1, 1.5)]))
        l.shadow_falloff_gamma = float(rng.uniform(0.5, 2))
    if kind in (RECT, DOME) and rng.random() < 0.5:
        l.texture = str(rng.choice(textures))
    return l


def fuzz_lights_box(seed: int, size: int = 40):
    """The closed box (its own or random materials) lit by one to six seeded
    random lights instead of its rect light."""
    import numpy as np

    from hdcodex_b200 import workloads
    rng = np.random.default_rng(10_000 + seed)
    wl = fuzz_box(seed, size) if rng.random() < 0.5 else workloads.closed_box(width=size, height=size, spp=4)
    s = wl.scene
    hdr = ("rect#hdr", "spectral-gradient#hdr")
    s.textures += [t for t in base_scene().textures if t.id in hdr]
    s.lights = [fuzz_light(rng, f"/light{i}", hdr) for i in range(int(rng.integers(1, 7)))]
    return wl


def _fuzz_texture(rng, texture_id: str) -> Texture:
    import numpy as np
    w, h = int(rng.integers(1, 9)), int(rng.integers(1, 9))
    kind = int(rng.integers(0, 3))  # sRGB8, linear RGBA8, RGBA32F
    if kind == 2:
        return Texture(id=texture_id, source_path="synthetic", width=w, height=h,
                       rgba_float=rng.uniform(0, 1.5, w * h * 4).astype(np.float32).tolist())
    return Texture(id=texture_id, source_path="synthetic", width=w, height=h, srgb=kind == 0,
                   rgba=rng.integers(0, 256, w * h * 4).tolist())


def _fuzz_normal_map(rng, texture_id: str) -> Texture:
    import numpy as np
    w, h = int(rng.integers(1, 6)), int(rng.integers(1, 6))
    n = rng.normal(size=(w * h, 3)) * 0.3 + np.array([0.0, 0.0, 1.0])
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    rgb = np.clip((n * 0.5 + 0.5) * 255, 0, 255).astype(int)
    return Texture(id=texture_id, source_path="synthetic", width=w, height=h,
                   rgba=np.concatenate([rgb, np.full((w * h, 1), 255)], axis=1).ravel().tolist())


def fuzz_textured(seed: int) -> Scene:
    """The reference's textured triangle with random UVs above a UV-tiled
    ground quad, both with random materials whose texture slots (all but
    opacity) bind seeded random textures (sRGB8, linear RGBA8, RGBA32F, at
    random a UDIM set of three tiles), a random normal map, and random
    base-colour scale, bias and channel."""
    import numpy as np

    from hdcodex_b200 import _abi
    rng = np.random.default_rng(20_000 + seed)
    s = base_scene()
    s.meshes.append(Mesh(id="/ground", positions=[-4, -1.0, -1, 4, -1.0, -1, 4, -1.0, -6, -4, -1.0, -6],
                         indices=[0, 1, 2, 0, 2, 3],
                         texcoords=[0.0, 0.0, 3.0, 0.0, 3.0, 2.5, 0.0, 0.0, 3.0, 2.5, 0.0, 2.5],
                         material_id="/groundMat"))
    s.meshes[0].texcoords = rng.uniform(-0.5, 2.5, 6).tolist()
    textures = [_fuzz_texture(rng, f"fuzz{i}") for i in range(4)] + [_fuzz_normal_map(rng, "fuzzNormal")]
    bindable = [t.id for t in textures if t.id != "fuzzNormal"]
    if rng.random() < 0.4:
        for tile in (1001, 1002, 1011):
            t = _fuzz_texture(rng, f"fuzzUdim#udim={tile}")
            t.udim_set_id, t.udim_tile, t.source_path = "fuzzUdim", tile, f"fuzzUdim.{tile}"
            textures.append(t)
        bindable.append("fuzzUdim")
    s.textures += textures
    slots = [n for n, _t, _d in _abi.MATERIAL_FIELDS if n.endswith("_texture") and n != "opacity_texture"]
    s.materials = []
    for material_id in ("/red", "/groundMat"):
        m = fuzz_material(rng, material_id)
        for slot in slots:
            if slot == "normal_texture":
                if rng.random() < 0.4:
                    m.normal_texture = "fuzzNormal"
                    m.normal_texture_scale = float(rng.uniform(0.2, 1.5))
                    m.normal_texture_flip_y = bool(rng.random() < 0.5)
            elif rng.random() < 0.3:
                setattr(m, slot, str(rng.choice(bindable)))
        if rng.random() < 0.5:
            m.base_color_texture_scale = rng.uniform(0.5, 1.5, 3).tolist()
            m.base_color_texture_bias = rng.uniform(-0.1, 0.2, 3).tolist()
            m.base_color_texture_channel = int(rng.integers(-1, 4))
        s.materials.append(m)
    return s
