"""The autotuner (hdcx_autotune) and launch tuning: the picked configuration
renders the same image as the defaults, bit for bit, and a repeated tuning of
the same workload shape is served from the process-wide cache."""
import numpy as np
import pytest

from hdcodex_b200 import PathTracer, workloads

pytestmark = pytest.mark.gpu


def test_autotune_picks_a_configuration_with_identical_images():
    wl = workloads.closed_box(width=96, height=96)
    with PathTracer(0) as t:
        t.set_scene(wl.scene)
        r = t.autotune(wl.camera, 96, 96, 8, 4)
        assert r["candidates"] >= 3 and r["milliseconds"] > 0 and r["milliseconds"] <= r["default_milliseconds"]
        assert t.tuning()["trace_blocks_per_sm"] == r["trace_blocks_per_sm"]
        tuned = t.render(wl.camera, 96, 96, 0, 8, 4)
    with PathTracer(0) as d:
        d.set_scene(wl.scene)
        default = d.render(wl.camera, 96, 96, 0, 8, 4)
        # Extreme launch shapes render the same image too.
        d.set_tuning(wave_paths=1000, trace_blocks_per_sm=1, shade_blocks_per_sm=64)
        odd = d.render(wl.camera, 96, 96, 0, 8, 4)
        again = d.autotune(wl.camera, 96, 96, 8, 4)  # same shape: from the cache
    assert np.array_equal(tuned, default) and np.array_equal(odd, default)
    assert again["candidates"] == 0 and again["trace_blocks_per_sm"] == r["trace_blocks_per_sm"]


def test_tuning_rejects_out_of_range_values():
    wl = workloads.closed_box(width=16, height=16)
    with PathTracer(0) as t:
        t.set_scene(wl.scene)
        with pytest.raises(RuntimeError, match="tuning out of range"):
            t.set_tuning(trace_blocks_per_sm=0)
        with pytest.raises(RuntimeError, match="tuning out of range"):
            t.set_tuning(wave_paths=2)
        with pytest.raises(RuntimeError, match="tuning out of range"):
            t.set_tuning(sort_hits=2)


def test_wave_size_follows_the_tuning_after_larger_buffers():
    """Path buffers are kept when a later call needs fewer paths, but each call
    launches waves of its own size: a smaller wave set after a large render
    takes effect (more waves, more launches) and renders the same image."""
    wl = workloads.closed_box(width=64, height=64)
    with PathTracer(0) as t:
        t.set_scene(wl.scene)
        one_wave = t.render(wl.camera, 64, 64, 0, 8, 4)  # 49,152 paths: one wave
        launches_one = t.stats()["kernel_launches"]
        t.set_tuning(wave_paths=4096)
        many_waves = t.render(wl.camera, 64, 64, 0, 8, 4)
        launches_many = t.stats()["kernel_launches"]
    assert np.array_equal(one_wave, many_waves)
    assert launches_many > 8 * launches_one, (launches_one, launches_many)


@pytest.mark.parametrize("make", [
    lambda: workloads.spectral_stress(width=96, height=54, spp=2, dome_size=(128, 64)),
    lambda: workloads.heavy_geometry(width=96, height=54, spp=2, dome_size=(128, 64)),
], ids=["stress", "heavy"])
def test_material_sorted_hits_render_the_same_image(make):
    """sort_hits shades each bounce's hits in material order (a counting sort
    of the hit queue); per-path results do not depend on the order."""
    wl = make()
    with PathTracer(0) as t:
        t.set_scene(wl.scene)
        t.set_tuning(wave_paths=8192)  # several waves per frame
        plain = t.render(wl.camera, wl.width, wl.height, 0, 8, wl.spp)
        plain_stats = t.stats()
        t.set_tuning(wave_paths=8192, sort_hits=1)
        assert t.tuning()["sort_hits"] == 1
        sorted_ = t.render(wl.camera, wl.width, wl.height, 0, 8, wl.spp)
        sorted_stats = t.stats()
    assert np.array_equal(plain, sorted_)
    for key in ("extension_rays", "shadow_rays", "subsurface_rays"):
        assert plain_stats[key] == sorted_stats[key], key
    assert sorted_stats["kernel_launches"] > plain_stats["kernel_launches"]


@pytest.mark.parametrize("make", [
    lambda: workloads.spectral_stress(width=96, height=54, spp=2, dome_size=(128, 64)),
    lambda: workloads.heavy_geometry(width=96, height=54, spp=2, dome_size=(128, 64)),
], ids=["stress", "heavy"])
def test_direction_sorted_rays_render_the_same_image(make):
    """sort_rays reorders each secondary extension queue by direction cell
    within chunks of 1024 entries; per-path results do not depend on the
    order, with or without the hit sort."""
    wl = make()
    with PathTracer(0) as t:
        t.set_scene(wl.scene)
        t.set_tuning(wave_paths=8192)
        plain = t.render(wl.camera, wl.width, wl.height, 0, 8, wl.spp)
        plain_stats = t.stats()
        for sort_hits in (0, 1):
            t.set_tuning(wave_paths=8192, sort_hits=sort_hits, sort_rays=1)
            assert t.tuning()["sort_rays"] == 1
            img = t.render(wl.camera, wl.width, wl.height, 0, 8, wl.spp)
            st = t.stats()
            assert np.array_equal(plain, img), sort_hits
            for key in ("extension_rays", "shadow_rays", "subsurface_rays"):
                assert plain_stats[key] == st[key], key
        with pytest.raises(RuntimeError, match="tuning out of range"):
            t.set_tuning(sort_rays=2)
