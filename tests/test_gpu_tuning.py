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
