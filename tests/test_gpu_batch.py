"""hdcx_render_batch: several jobs rendered together equal the same jobs
rendered one hdcx_render call at a time, bit for bit (images, running means
and counters), whatever wave size each job runs with, launched on the jobs'
streams or captured into one CUDA graph (HDCX_BATCH_CUDA_GRAPH)."""
import numpy as np
import pytest

import ref_scenes as R
from hdcodex_b200 import PathTracer, render_batch, workloads

pytestmark = pytest.mark.gpu

INVALID_ARGUMENT = 1


def jobs_spec():
    heavy = workloads.heavy_geometry(width=160, height=90, spp=3, dome_size=(256, 128))
    stress = workloads.spectral_stress(width=96, height=54, spp=2, dome_size=(128, 64))
    box = workloads.closed_box(width=128, height=128, spp=4)
    small = workloads.batch_job(2)
    return [
        (R.base_scene(), R.base_camera(), 64, 64, 5),
        (box.scene, box.camera, box.width, box.height, box.spp),
        (heavy.scene, heavy.camera, heavy.width, heavy.height, heavy.spp),
        (stress.scene, stress.camera, stress.width, stress.height, stress.spp),
        (small.scene, small.camera, 128, 96, 2),
    ]


@pytest.fixture(scope="module")
def sequential():
    """Reference images: one hdcx_render per job, two progressive calls each."""
    out = []
    for scene, cam, w, h, spp in jobs_spec():
        with PathTracer(0) as t:
            t.set_scene(scene)
            first = t.render(cam, w, h, 0, 8, spp)
            stats_first = t.stats()
            second = t.render(cam, w, h, spp, 8, 2)
            out.append((first, second, stats_first))
    return out


@pytest.mark.parametrize("wave,graph", [(0, False), (5000, False), (0, True), (5000, True)])
def test_batch_equals_sequential(sequential, wave, graph):
    spec = jobs_spec()
    tracers = [PathTracer(0) for _ in spec]
    budget = 0
    try:
        for t, (scene, *_rest) in zip(tracers, spec):
            t.set_scene(scene)
            t.set_wave_size(wave)  # 5000: many small waves per job
        images = [np.zeros((h, w, 4), np.float32) for _, _, w, h, _ in spec]
        jobs = [(t, cam, w, h, 0, 8, spp, img) for t, (_, cam, w, h, spp), img in zip(tracers, spec, images)]
        results = render_batch(jobs, budget, graph=graph)
        assert all(r["written"] == 1 and r["status"] == 0 and r["render_ms"] > 0 for r in results)
        for k, (img, t) in enumerate(zip(images, tracers)):
            first, _, stats = sequential[k]
            assert np.array_equal(img, first), f"job {k}: identical={np.all(img == first, axis=-1).mean():.4f}"
            got = t.stats()
            for key in ("spectral_paths", "extension_rays", "shadow_rays", "subsurface_rays"):
                assert got[key] == stats[key], (k, key)
        # A second, progressive batch on top of the first.
        images2 = [np.zeros_like(img) for img in images]
        jobs = [(t, cam, w, h, spp, 8, 2, img) for t, (_, cam, w, h, spp), img in zip(tracers, spec, images2)]
        render_batch(jobs, budget, graph=graph)
        for k, img in enumerate(images2):
            assert np.array_equal(img, sequential[k][1]), f"job {k} progressive"
    finally:
        for t in tracers:
            t.close()


def test_batch_rejects_a_tracer_twice():
    from hdcodex_b200 import _abi
    from hdcodex_b200.tracer import lib
    with PathTracer(0) as t:
        t.set_scene(R.base_scene())
        arr = (_abi.BatchJob * 2)()
        for b in arr:
            b.tracer = t.handle
            b.camera = R.base_camera()
            b.width = b.height = 8
            b.sample_count = 1
            b.max_bounces = 8
        assert lib().hdcx_render_batch(arr, 2, 0) == INVALID_ARGUMENT
        assert b"more than one job" in lib().hdcx_last_error(t.handle)
        assert lib().hdcx_render_batch(arr, 0, 0) == 0
        assert lib().hdcx_render_batch(None, 1, 0) == INVALID_ARGUMENT


def test_batch_job_without_geometry_writes_nothing():
    with PathTracer(0) as empty, PathTracer(0) as full:
        full.set_scene(R.base_scene())
        a = np.zeros((16, 16, 4), np.float32)
        b = np.zeros((16, 16, 4), np.float32)
        results = render_batch([(empty, R.base_camera(), 16, 16, 0, 8, 1, a),
                                (full, R.base_camera(), 16, 16, 0, 8, 1, b)])
        assert results[0]["written"] == 0 and results[0]["status"] == 0
        assert results[1]["written"] == 1
        assert not a.any() and b[..., 3].min() == 1.0


@pytest.mark.parametrize("graph", [False, True])
def test_jobs_sharing_lane_buffers_equal_sequential(graph):
    """Eleven jobs: more than the batch's lanes, so several jobs render one
    after another on one lane's path buffers. Each job's image and counters
    equal its own hdcx_render call."""
    spec = [(workloads.closed_box(width=w, height=h, spp=spp), w, h, spp)
            for w, h, spp in [(96, 64, 3), (64, 64, 2), (128, 72, 1), (80, 80, 4), (32, 48, 5), (72, 40, 2),
                              (100, 60, 2), (48, 48, 6), (120, 90, 1), (56, 72, 3), (64, 32, 7)]]
    expected = []
    for wl, w, h, spp in spec:
        with PathTracer(0) as t:
            t.set_scene(wl.scene)
            expected.append((t.render(wl.camera, w, h, 0, 8, spp), t.stats()))
    tracers = [PathTracer(0) for _ in spec]
    try:
        for t, (wl, *_rest) in zip(tracers, spec):
            t.set_scene(wl.scene)
        images = [np.zeros((h, w, 4), np.float32) for _, w, h, _ in spec]
        jobs = [(t, wl.camera, w, h, 0, 8, spp, img) for t, (wl, w, h, spp), img in zip(tracers, spec, images)]
        results = render_batch(jobs, 0, graph=graph)
        assert all(r["written"] == 1 and r["status"] == 0 for r in results)
        for k, (img, t) in enumerate(zip(images, tracers)):
            ref, stats = expected[k]
            assert np.array_equal(img, ref), k
            got = t.stats()
            for key in ("spectral_paths", "extension_rays", "shadow_rays"):
                assert got[key] == stats[key], (k, key)
    finally:
        for t in tracers:
            t.close()


def test_batch_graph_is_updated_in_place_and_times_jobs():
    """A second batch with the same launch topology updates the device's cached
    executable graph (cudaGraphExecUpdate) instead of instantiating a new one;
    the images still equal one hdcx_render per job, and each job reports its
    own device time inside the graph (at most the whole batch's time)."""
    from hdcodex_b200.tracer import batch_graph_stats
    spec = [(workloads.closed_box(width=w, height=h, spp=spp), w, h, spp)
            for w, h, spp in [(64, 48, 2), (96, 64, 3), (32, 32, 4)]]
    tracers = [PathTracer(0) for _ in spec]
    try:
        for t, (wl, *_rest) in zip(tracers, spec):
            t.set_scene(wl.scene)
        images = [np.zeros((h, w, 4), np.float32) for _, w, h, _ in spec]
        for call, sample_index in enumerate((0, 7)):
            before = batch_graph_stats(0)
            jobs = [(t, wl.camera, w, h, sample_index, 8, spp, img)
                    for t, (wl, w, h, spp), img in zip(tracers, spec, images)]
            results = render_batch(jobs, 0, graph=True)
            after = batch_graph_stats(0)
            assert all(r["status"] == 0 and r["written"] == 1 for r in results)
            if call == 1:
                assert after[1] == before[1] + 1 and after[0] == before[0], (before, after)
            ms = [r["render_ms"] for r in results]
            assert all(m > 0 for m in ms)
        for k, (wl, w, h, spp) in enumerate(spec):
            with PathTracer(0) as ref:
                ref.set_scene(wl.scene)
                ref.render(wl.camera, w, h, 0, 8, spp)
                expected = ref.render(wl.camera, w, h, 7, 8, spp)
            assert np.array_equal(images[k], expected), k
    finally:
        for t in tracers:
            t.close()
