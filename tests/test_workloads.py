"""The seeded synthetic workloads have the shapes of the benchmark configs:
C1 closed box (34 triangles, 256x256, 16 spp), C2 heavy geometry (1,000,480
triangles, 1920x1080, 64 spp), C3 spectral stress (~200k triangles,
1280x720, 256 spp), C4 64 jobs (triangles log-uniform in [10k, 2M],
resolutions from the four sizes, spp in 4..128, a dome and 1-8 lights), all
with 8 bounces; and they are pure functions of their seeds."""
import numpy as np

from hdcodex_b200 import workloads as W


def paths(wl):
    return wl.width * wl.height * wl.spp * 3


def test_closed_box_shape():
    wl = W.closed_box()
    assert W.triangle_count(wl.scene) == 34
    assert (wl.width, wl.height, wl.spp, wl.max_bounces) == (256, 256, 16, 8)
    assert paths(wl) == 3_145_728 == wl.spectral_paths


def test_heavy_geometry_shape():
    wl = W.heavy_geometry()
    assert W.triangle_count(wl.scene) == 1_000_480
    assert (wl.width, wl.height, wl.spp, wl.max_bounces) == (1920, 1080, 64, 8)
    assert paths(wl) == 398_131_200 == wl.spectral_paths
    dome = [t for t in wl.scene.textures if t.rgba_float is not None]
    assert any((t.width, t.height) == (2048, 1024) for t in dome)


def test_spectral_stress_shape():
    wl = W.spectral_stress()
    assert 190_000 <= W.triangle_count(wl.scene) <= 210_000
    assert (wl.width, wl.height, wl.spp, wl.max_bounces) == (1280, 720, 256, 8)
    assert paths(wl) == 707_788_800 == wl.spectral_paths
    m = wl.scene.materials
    assert any(x.transmission > 0 and x.transmission_dispersion_scale > 0 for x in m)
    assert any(x.subsurface > 0 for x in m)
    assert any(x.opacity_texture for x in m)


def test_batch_jobs_follow_the_distribution():
    jobs = W.batch_jobs(64)
    tris = np.array([W.triangle_count(j.scene) for j in jobs])
    assert tris.min() >= 9_000 and tris.max() <= 2_100_000
    # Log-uniform: a spread over two decades, not clustered at either end.
    assert np.log10(tris.max() / tris.min()) > 1.5
    assert {(j.width, j.height) for j in jobs} <= set(W.BATCH_RESOLUTIONS)
    assert all(4 <= j.spp <= 128 and j.max_bounces == 8 for j in jobs)
    assert all(2 <= len(j.scene.lights) <= 9 for j in jobs)  # the dome and 1-8 analytic lights


def test_workloads_are_pure_functions_of_their_seeds():
    a, b = W.batch_job(3), W.batch_job(3)
    assert (a.width, a.height, a.spp) == (b.width, b.height, b.spp)
    for ma, mb in zip(a.scene.meshes, b.scene.meshes):
        assert np.array_equal(np.asarray(ma.positions), np.asarray(mb.positions))
        assert np.array_equal(np.asarray(ma.indices), np.asarray(mb.indices))
    c = W.batch_job(3, seed=1)
    assert not all(np.array_equal(np.asarray(x.positions), np.asarray(y.positions))
                   for x, y in zip(a.scene.meshes, c.scene.meshes))
    s1, s2 = W.spectral_stress(width=64, height=36), W.spectral_stress(width=64, height=36)
    assert np.array_equal(np.asarray(s1.scene.meshes[0].positions), np.asarray(s2.scene.meshes[0].positions))
