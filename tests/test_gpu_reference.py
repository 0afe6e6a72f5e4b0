"""The reference's own test expectations (tests/path_tracer_tests.cpp of
hdCodex) on the CUDA tracer: the same scenes, sample counts and thresholds as
tests/test_oracle_reference.py, run through the C ABI."""
import pytest

import test_oracle_reference as checks
from hdcodex_b200 import PathTracer

pytestmark = pytest.mark.gpu


class _GpuBackend:
    @staticmethod
    def OracleTracer():
        return PathTracer(0)


@pytest.fixture(scope="module")
def gpu_backend():
    return _GpuBackend


@pytest.fixture(scope="module")
def gpu_base_image(gpu_backend):
    return checks.render(gpu_backend, checks.R.base_scene(), 64)


def test_batched_equals_sequential(gpu_backend):
    checks.test_batched_equals_sequential(gpu_backend)


def test_base_image(gpu_base_image):
    checks.test_base_image(gpu_base_image)


@pytest.mark.parametrize("index", range(4))
def test_analytic_lights_illuminate(gpu_backend, index):
    checks.test_analytic_lights_illuminate(gpu_backend, index)


def test_power_weighted_selection(gpu_backend):
    checks.test_power_weighted_selection(gpu_backend)


def test_mesh_light_nee(gpu_backend):
    checks.test_mesh_light_nee(gpu_backend)


def test_oren_nayar_changes_image(gpu_backend, gpu_base_image):
    checks.test_oren_nayar_changes_image(gpu_backend, gpu_base_image)


def test_udim_tile_selected(gpu_backend):
    checks.test_udim_tile_selected(gpu_backend)


def test_progressive_and_interactive_sizes(gpu_backend):
    checks.test_progressive_and_interactive_sizes(gpu_backend)


def test_authored_normals(gpu_backend, gpu_base_image):
    checks.test_authored_normals(gpu_backend, gpu_base_image)


def test_ggx_and_coat_highlights(gpu_backend):
    checks.test_ggx_and_coat_highlights(gpu_backend)


def test_subsurface_tints_blue(gpu_backend):
    checks.test_subsurface_tints_blue(gpu_backend)


def test_cutout_reveals_environment(gpu_backend):
    checks.test_cutout_reveals_environment(gpu_backend)


def test_translucent_backlighting(gpu_backend):
    checks.test_translucent_backlighting(gpu_backend)


def test_thin_walled_tint(gpu_backend):
    checks.test_thin_walled_tint(gpu_backend)


def test_dispersion_changes_image(gpu_backend):
    checks.test_dispersion_changes_image(gpu_backend)


def test_fallback_sun_and_sky(gpu_backend):
    checks.test_fallback_sun_and_sky(gpu_backend)


def test_no_geometry_returns_nothing(gpu_backend):
    checks.test_no_geometry_returns_nothing(gpu_backend)


def test_shading_modes(gpu_backend):
    t = PathTracer(0)
    assert t.get_shading_mode() == 0
    t.set_shading_mode(1)
    assert t.get_shading_mode() == 1
    with pytest.raises(ValueError):
        t.set_shading_mode(2)
    t.set_shading_mode(0)
