"""The CPU oracle against the reference's own test expectations.

tests/path_tracer_tests.cpp of hdCodex checks its Vulkan integrator with one
exact check (two sequential 1-spp renders equal one batched 2-spp render
within 1e-5, :143-150) and a list of qualitative inequalities on a triangle
scene. The same checks, with the same scenes, sample counts and thresholds,
pin the oracle's restatement of the integrator."""
import numpy as np
import pytest

import ref_scenes as R

W, H = R.WIDTH, R.HEIGHT
CY, CX = R.CENTER


def luma(img, y, x):
    return float(img[y, x, 0] + img[y, x, 1] + img[y, x, 2])


def render(oracle_lib, scene, spp, camera=None, tracer=None, bounces=8):
    t = tracer or oracle_lib.OracleTracer()
    t.set_scene(scene)
    return t.render(camera or R.base_camera(), W, H, 0, bounces, spp)


@pytest.fixture(scope="module")
def base_image(oracle_lib):
    return render(oracle_lib, R.base_scene(), 64)


def test_batched_equals_sequential(oracle_lib):
    # path_tracer_tests.cpp:140-150
    t = oracle_lib.OracleTracer()
    t.set_scene(R.base_scene())
    cam = R.base_camera()
    first = t.render(cam, W, H, 0)
    second = t.render(cam, W, H, 1)
    batched = t.render(cam, W, H, 0, 8, 2)
    assert first.shape == batched.shape
    assert np.abs(batched - second).max() < 1e-5


def test_base_image(base_image):
    # :152-166
    assert base_image.shape == (H, W, 4)
    assert np.isfinite(base_image).all()
    assert abs(luma(base_image, CY, CX) - luma(base_image, 0, 0)) > 0.02
    assert base_image[CY, CX, 1] > base_image[CY, CX, 0] * 1.5
    assert base_image[CY, CX, 3] == 1.0


@pytest.mark.parametrize("index", range(4))
def test_analytic_lights_illuminate(oracle_lib, index):
    # :169-215
    s = R.base_scene()
    s.lights = [R.analytic_lights()[index]]
    img = render(oracle_lib, s, 32)
    c = luma(img, CY, CX)
    assert np.isfinite(c) and c > 0.01


def test_power_weighted_selection(oracle_lib):
    # :217-232
    img = render(oracle_lib, R.selection_scene(), 1)
    c = luma(img, CY, CX)
    assert np.isfinite(c) and c > 0.01


def test_mesh_light_nee(oracle_lib):
    # :237-291
    lit = render(oracle_lib, R.mesh_light_scene(1.0), 32)
    dark = render(oracle_lib, R.mesh_light_scene(0.0), 32)
    assert luma(lit, CY, CX) > luma(dark, CY, CX) + 0.02


def test_oren_nayar_changes_image(oracle_lib, base_image):
    # :294-311
    rough = render(oracle_lib, R.variant("oren_nayar"), 64)
    assert np.abs(rough[..., :3] - base_image[..., :3]).sum() > 0.05


def test_udim_tile_selected(oracle_lib):
    # :313-326
    img = render(oracle_lib, R.variant("udim"), 64)
    assert img[CY, CX, 2] > img[CY, CX, 0] * 2.0


def test_progressive_and_interactive_sizes(oracle_lib):
    # :328-332
    t = oracle_lib.OracleTracer()
    t.set_scene(R.base_scene())
    cam = R.base_camera()
    assert t.render(cam, W, H, 0, 8, 64).shape == (H, W, 4)
    assert t.render(cam, W, H, 64).shape == (H, W, 4)
    small = t.render(cam, W // 2, H // 2, 0, 2)
    assert small.size == W * H


def test_authored_normals(oracle_lib, base_image):
    # :334-343
    img = render(oracle_lib, R.variant("authored_normals"), 64)
    assert abs(img[CY, CX, 1] - base_image[CY, CX, 1]) > 0.02


def test_ggx_and_coat_highlights(oracle_lib):
    # :345-371
    glossy = render(oracle_lib, R.variant("glossy"), 64)
    matte = render(oracle_lib, R.variant("matte_black"), 64)
    coated = render(oracle_lib, R.variant("coated"), 64)
    assert luma(glossy, CY, CX) > luma(matte, CY, CX) + 0.1
    assert luma(coated, CY, CX) > luma(matte, CY, CX) + 0.1


def test_subsurface_tints_blue(oracle_lib):
    # :373-386
    img = render(oracle_lib, R.variant("subsurface"), 64)
    assert img[CY, CX, 2] > img[CY, CX, 1] * 1.5


def test_cutout_reveals_environment(oracle_lib):
    # :391-395
    img = render(oracle_lib, R.variant("cutout"), 64)
    assert img[CY, CX, 2] > img[CY, CX, 1]


def test_translucent_backlighting(oracle_lib):
    # :397-414
    black = render(oracle_lib, R.variant("opaque_black"), 64)
    tr = render(oracle_lib, R.variant("translucent"), 64)
    assert tr[CY, CX, 0] > tr[CY, CX, 1] * 2.0
    assert luma(tr, CY, CX) > luma(black, CY, CX) + 0.01


def test_thin_walled_tint(oracle_lib):
    # :416-426
    img = render(oracle_lib, R.variant("thin_walled"), 64)
    assert img[CY, CX, 0] > img[CY, CX, 1] * 2.0


def test_dispersion_changes_image(oracle_lib):
    # :428-449
    a = render(oracle_lib, R.variant("nondispersive"), 64)
    b = render(oracle_lib, R.variant("dispersive"), 64)
    assert np.abs(a[..., :3] - b[..., :3]).sum() > 0.1


def test_fallback_sun_and_sky(oracle_lib):
    # :451-490
    img = render(oracle_lib, R.variant("fallback"), 64)
    assert luma(img, CY, CX) > 0.05
    assert img[CY, CX, 1] > img[CY, CX, 0] * 2.0
    assert luma(img, 0, 0) > 0.05
    zup = oracle_lib.OracleTracer()
    zimg = render(oracle_lib, R.variant("fallback_zup"), 64, camera=R.z_up_camera(), tracer=zup)
    assert luma(zimg, CY, CX) > 0.05


def test_no_geometry_returns_nothing(oracle_lib):
    t = oracle_lib.OracleTracer()
    assert t.render(R.base_camera(), W, H, 0) is None
    t.set_scene(R.base_scene())
    assert t.has_geometry()
    assert t.render(R.base_camera(), 0, H, 0) is None
