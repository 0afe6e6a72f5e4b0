"""Path state lives in per-device arenas that renders check out for their
duration (hdcx_api.cpp, "Path arenas"): tracers that render one after another
share them, renders on several host threads take separate arenas or wait for
one, and every image equals the one a fresh tracer renders alone, bit for bit."""
import threading

import numpy as np
import pytest

import ref_scenes as R
from hdcodex_b200 import PathTracer, workloads

pytestmark = pytest.mark.gpu


def cases():
    box = workloads.closed_box(width=96, height=64, spp=3)
    heavy = workloads.heavy_geometry(width=80, height=48, spp=2, dome_size=(128, 64))
    return [
        (R.base_scene(), R.base_camera(), 64, 64, 4),
        (box.scene, box.camera, box.width, box.height, box.spp),
        (heavy.scene, heavy.camera, heavy.width, heavy.height, heavy.spp),
    ]


@pytest.fixture(scope="module")
def alone():
    out = []
    for scene, cam, w, h, spp in cases():
        with PathTracer(0) as t:
            t.set_scene(scene)
            first = t.render(cam, w, h, 0, 8, spp)
            out.append((first, t.render(cam, w, h, spp, 8, spp)))
    return out


def test_tracers_rendering_in_turn_share_arenas(alone):
    spec = cases()
    tracers = [PathTracer(0) for _ in spec]
    try:
        for t, (scene, *_rest) in zip(tracers, spec):
            t.set_scene(scene)
        # Interleaved progressive renders: each call may take an arena another
        # tracer used (and grew) before it.
        first = [t.render(cam, w, h, 0, 8, spp) for t, (_, cam, w, h, spp) in zip(tracers, spec)]
        second = [t.render(cam, w, h, spp, 8, spp) for t, (_, cam, w, h, spp) in zip(tracers, spec)]
        for k in range(len(spec)):
            assert np.array_equal(first[k], alone[k][0]), k
            assert np.array_equal(second[k], alone[k][1]), k
    finally:
        for t in tracers:
            t.close()


def test_concurrent_renders_on_host_threads(alone):
    spec = cases()
    results = {}
    errors = []

    def work(k, repeats):
        scene, cam, w, h, spp = spec[k]
        try:
            with PathTracer(0) as t:
                t.set_scene(scene)
                for _ in range(repeats):
                    a = t.render(cam, w, h, 0, 8, spp)
                    b = t.render(cam, w, h, spp, 8, spp)
                results[k] = (a, b)
        except Exception as e:  # reported below, on the main thread
            errors.append((k, repr(e)))

    threads = [threading.Thread(target=work, args=(k, 3)) for k in range(len(spec))]
    for th in threads:
        th.start()
    for th in threads:
        th.join(timeout=300)
    assert not any(th.is_alive() for th in threads), "a render thread did not finish"
    assert not errors, errors
    for k in range(len(spec)):
        assert np.array_equal(results[k][0], alone[k][0]), k
        assert np.array_equal(results[k][1], alone[k][1]), k
