"""Texture level of detail (hdcx_set_texture_lod), which the reference does
not have (its sampler reads one mip level; README.md lists texture LOD as
future work). The reference's images are the LOD-off images, which every
parity test pins; here:

* the mip pyramid the GPU builds equals a numpy restatement of its rule (2x2
  means in binary32, ((a + b) + (c + d)) * 0.25, odd sizes reusing their last
  row or column) bit for bit, for RGBA32F and RGBA8 textures of odd sizes;
* turning LOD off again gives the reference's images bit for bit;
* on a finely checkered ground plane seen at a grazing angle and lit by one
  sharp distant light (direct light only, so that the per-pixel variance is
  the texture's, not the lighting's), low-spp renders with LOD are closer to
  the converged image than renders without (less aliasing noise), measured
  on luminance.
"""
import numpy as np
import pytest

from hdcodex_b200 import DISTANT, Light, Material, Mesh, PathTracer, Scene, Texture, workloads

pytestmark = pytest.mark.gpu


def numpy_pyramid(level0):
    levels = [level0]
    cur = level0
    while cur.shape[0] > 1 or cur.shape[1] > 1:
        h, w = cur.shape[:2]
        nh, nw = max(1, h >> 1), max(1, w >> 1)
        ys0 = np.minimum(2 * np.arange(nh), h - 1)
        ys1 = np.minimum(2 * np.arange(nh) + 1, h - 1)
        xs0 = np.minimum(2 * np.arange(nw), w - 1)
        xs1 = np.minimum(2 * np.arange(nw) + 1, w - 1)
        a, b = cur[ys0][:, xs0], cur[ys0][:, xs1]
        c, d = cur[ys1][:, xs0], cur[ys1][:, xs1]
        cur = (((a + b) + (c + d)) * np.float32(0.25)).astype(np.float32)
        levels.append(cur)
    return levels


def textured_quad_scene(textures):
    s = Scene(revision=1)
    s.meshes.append(Mesh(id="/quad", positions=[-1, -1, -3, 1, -1, -3, 1, 1, -3, -1, 1, -3],
                         indices=[0, 1, 2, 0, 2, 3], texcoords=[0, 0, 1, 0, 1, 1, 0, 0, 1, 1, 0, 1],
                         material_id="/m"))
    s.materials.append(Material(id="/m", base_color_texture=textures[0].id, roughness_texture=textures[-1].id))
    s.textures += textures
    return s


def test_mip_pyramid_matches_numpy():
    rng = np.random.default_rng(1)
    f32 = rng.uniform(0, 4, (21, 37, 4)).astype(np.float32)
    u8 = rng.integers(0, 256, (33, 18, 4)).astype(np.uint8)
    textures = [Texture(id="f#hdr", width=37, height=21, rgba_float=f32.ravel()),
                Texture(id="u#raw", width=18, height=33, srgb=False, rgba=u8.ravel())]
    with PathTracer(0) as t:
        t.set_scene(textured_quad_scene(textures))
        t.set_texture_lod(1)
        for index, level0 in ((0, f32), (1, (u8.astype(np.float32) / np.float32(255.0)).astype(np.float32))):
            expected = numpy_pyramid(level0)
            for level in range(1, len(expected)):
                got = t.texture_level(index, level)
                assert got.shape == expected[level].shape, (index, level)
                assert np.array_equal(got, expected[level]), (index, level)
            with pytest.raises(RuntimeError, match="no such mip level"):
                t.texture_level(index, len(expected))
        with pytest.raises(RuntimeError):
            t.set_texture_lod(2)


def checker_ground(repeats=400.0, sun=False):
    """A large ground plane with a 1-texel checker repeated many times, seen
    from just above at a grazing angle, lit by the fallback sun and sky, or
    (sun=True) by one distant light from straight above with no angular size
    (its light sample has no randomness)."""
    n = 64
    checker = ((np.add.outer(np.arange(n), np.arange(n)) & 1) * 235 + 10).astype(np.uint8)
    rgba = np.stack([checker, checker, checker, np.full_like(checker, 255)], -1)
    s = Scene(revision=1)
    r = repeats
    s.meshes.append(Mesh(id="/ground", positions=[-50, 0, -100, 50, 0, -100, 50, 0, 5, -50, 0, 5],
                         indices=[0, 2, 1, 0, 3, 2], texcoords=[0, 0, r, r, r, 0, 0, 0, 0, r, r, r],
                         material_id="/check"))
    s.materials.append(Material(id="/check", base_color=[1, 1, 1], base_color_texture="checker#raw",
                                specular_weight=0.0))
    s.textures.append(Texture(id="checker#raw", width=n, height=n, srgb=False, rgba=rgba.ravel()))
    if sun:
        s.lights.append(Light(id="/sun", type=DISTANT, intensity=3.0, angle=0.0, basis_x=[1.0, 0.0, 0.0],
                              basis_y=[0.0, 0.0, -1.0], basis_z=[0.0, 1.0, 0.0]))
    cam = workloads.look_at_camera((0.0, 1.0, 4.0), (0.0, 0.0, -30.0), (0.0, 1.0, 0.0), 40.0, 96 / 64)
    return s, cam


def test_lod_off_is_the_reference_sampling():
    s, cam = checker_ground()
    with PathTracer(0) as t:
        t.set_scene(s)
        ref = t.render(cam, 96, 64, 0, 2, 2).copy()
        t.set_texture_lod(1)
        lod = t.render(cam, 96, 64, 0, 2, 2).copy()
        t.set_texture_lod(0)
        again = t.render(cam, 96, 64, 0, 2, 2)
    assert np.array_equal(ref, again)
    assert not np.array_equal(ref, lod)


def test_lod_reduces_aliasing_at_low_sample_counts():
    """Progressive 1-spp passes of two tracers, one sampling the checker at
    one mip level (the reference's sampling) and one with ray-cone LOD, one
    bounce (direct light) under a sharp distant light: over the passes the
    LOD image is nearer the converged one. The error is measured on the
    luminance (Y of the FP64 XYZ sums): the three hero wavelengths of a
    sample make the RGB of a single sample noisy whatever the texture does
    (about the size of the aliasing here), Y much less so. Each tracer keeps
    its own running sums (a pass with sample index k > 0 adds to them)."""
    s, cam = checker_ground(sun=True)
    w, h = 96, 64

    def luminance(t):
        total, samples = t.read_xyz()
        return np.asarray(total)[..., 1] / max(samples, 1)

    with PathTracer(0) as t_off, PathTracer(0) as t_on:
        t_off.set_scene(s)
        t_on.set_scene(s)
        t_on.set_texture_lod(1)
        t_off.render(cam, w, h, 0, 1, 1024)
        truth = luminance(t_off).copy()
        ground = truth > 0.0
        err_off, err_on = [], []
        for index in range(4):
            t_off.render(cam, w, h, index, 1, 1)
            t_on.render(cam, w, h, index, 1, 1)
            err_off.append(float(np.sqrt(np.mean((luminance(t_off) - truth)[ground] ** 2))))
            err_on.append(float(np.sqrt(np.mean((luminance(t_on) - truth)[ground] ** 2))))
    assert ground.mean() > 0.3
    assert np.mean(err_on) < 0.8 * np.mean(err_off), (err_on, err_off)
