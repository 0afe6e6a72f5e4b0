"""The integrator with the radiance cache attached (hdcx_set_radiance_cache).

Paths stop after a 2-bounce prefix and take the cache's prediction; a sparse
set of full-length training paths trains the cache online, wave by wave. The
method without the network is the same 2-bounce prefix with nothing after it:
it loses the light of longer paths. The test measures both against a
high-spp plain render of the same scene."""
import numpy as np
import pytest

from hdcodex_b200 import PathTracer, RadianceCache, workloads

pytestmark = pytest.mark.gpu

W = H = 64


def rel_rmse(img, ref):
    return float(np.sqrt(np.mean((img[..., :3] - ref[..., :3]) ** 2)) / np.sqrt(np.mean(ref[..., :3] ** 2)))


@pytest.fixture(scope="module")
def box():
    return workloads.closed_box(width=W, height=H)


@pytest.fixture(scope="module")
def reference(box):
    with PathTracer(0) as t:
        t.set_scene(box.scene)
        return t.render(box.camera, W, H, 0, 8, 1024)


def test_cache_mode_renders_and_trains(box):
    with PathTracer(0) as t, RadianceCache(0, log2_table_size=16, finest_resolution=256) as cache:
        t.set_scene(box.scene)
        t.set_radiance_cache(cache, prefix_bounces=2, training_paths=2048, train_steps=1)
        img = t.render(box.camera, W, H, 0, 8, 4)
        st = t.radiance_cache_stats()
        assert np.isfinite(img).all() and img[..., 3].min() == 1.0
        assert st["queries"] > 0 and st["samples"] > 0 and np.isfinite(st["last_loss"])
        # Detached, the tracer is the plain integrator again, bit for bit.
        t.set_radiance_cache(None)
        plain = t.render(box.camera, W, H, 0, 8, 4)
    with PathTracer(0) as fresh:
        fresh.set_scene(box.scene)
        assert np.array_equal(plain, fresh.render(box.camera, W, H, 0, 8, 4))


def test_trained_cache_recovers_the_truncated_light(box, reference):
    spp = 64
    with PathTracer(0) as t:
        t.set_scene(box.scene)
        truncated = t.render(box.camera, W, H, 0, 2, spp)  # the 2-bounce prefix without the cache
    with PathTracer(0) as t, RadianceCache(0, log2_table_size=16, finest_resolution=256, seed=5) as cache:
        t.set_scene(box.scene)
        t.set_radiance_cache(cache, prefix_bounces=2, training_paths=4096, train_steps=2)
        for frame in range(48):  # online training, one wave per frame
            t.render(box.camera, W, H, frame, 8, 1)
        cached = None
        for frame in range(spp):
            cached = t.render(box.camera, W, H, frame, 8, 1)
    e_truncated = rel_rmse(truncated, reference)
    e_cached = rel_rmse(cached, reference)
    mean_ref = reference[..., :3].mean()
    assert truncated[..., :3].mean() < 0.95 * mean_ref  # the prefix alone is missing light
    assert e_cached < 0.6 * e_truncated, (e_cached, e_truncated)
    assert abs(cached[..., :3].mean() / mean_ref - 1.0) < 0.1


def test_spread_termination(box, reference):
    """Paths ended by the spread heuristic (Mueller et al. 2021): a factor
    that never triggers ends the same paths as the prefix alone;
    with the paper's c = 0.01 paths end at the first vertex after a diffuse
    bounce (in the all-diffuse box: nearly every path at bounce 1), and the
    trained cache recovers the light beyond the direct lighting."""
    def run(spread, frames=48, spp=32, prefix=2):
        with PathTracer(0) as t, RadianceCache(0, log2_table_size=16, finest_resolution=256, seed=5) as cache:
            t.set_scene(box.scene)
            t.set_radiance_cache(cache, prefix_bounces=prefix, training_paths=4096, train_steps=2)
            t.set_radiance_cache_spread(spread)
            for frame in range(frames):
                t.render(box.camera, W, H, frame, 8, 1)
            img = None
            for frame in range(spp):
                img = t.render(box.camera, W, H, frame, 8, 1)
            return img.copy(), t.radiance_cache_stats()

    prefix_only, st_prefix = run(0.0, frames=4, spp=4)
    never, st_never = run(1e6, frames=4, spp=4)
    # The same paths end at the same vertices; the images differ only by the
    # order of the training's atomic gradient sums (not bit-reproducible).
    assert st_prefix["queries"] == st_never["queries"]
    assert rel_rmse(never, prefix_only) < 1e-2
    spread, _ = run(0.01, prefix=4)
    assert np.isfinite(spread).all()
    with PathTracer(0) as t:
        t.set_scene(box.scene)
        direct = t.render(box.camera, W, H, 0, 1, 32)  # one bounce, no cache: direct light only
    assert rel_rmse(spread, reference) < 0.6 * rel_rmse(direct, reference)
    assert abs(spread[..., :3].mean() / reference[..., :3].mean() - 1.0) < 0.1
    with PathTracer(0) as t:
        with pytest.raises(RuntimeError):
            t.set_radiance_cache_spread(-1.0)
