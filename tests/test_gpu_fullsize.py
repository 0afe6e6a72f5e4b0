"""GPU parity at the configs' full sizes.

The CUDA tracer renders the whole frame of each config with the launch tuning
the benchmark runs it at; the oracle renders crops of the same frame (its
`crop=` renders only those pixels, with the same per-pixel seeds), and the
crops must agree at the parity tolerance of test_gpu_parity.py (at least 99%
of pixels bit-identical, image-level relative L1 difference at most 1e-3).

What only these sizes reach:
* the 1.0M-triangle scene with its full 2048x1024 dome: the dome's
  importance CDF of 2048x1024 texels and its 32-stride skip arrays
  (vulkan_path_tracer.cpp:583-650 dome sampling, :1998-2066 host CDF);
* 48M-path waves (six spp of a 1080p frame per wave), the autotuner's pick
  for that scene, and the stress scene's material-sorted hit queue
  (`sort_hits`) at 1280x720;
* the closed box at 256x256 and 16 spp, its config in full.
"""
import numpy as np
import pytest

from hdcodex_b200 import PathTracer, workloads

pytestmark = pytest.mark.gpu

MIN_IDENTICAL = 0.99
MAX_REL_L1 = 1e-3
SIDE = 64


@pytest.fixture(scope="module")
def gpu():
    t = PathTracer(0)
    yield t
    t.close()


def crops(width, height):
    """Five SIDE x SIDE crops: the centre and one in each quadrant."""
    out = [((width - SIDE) // 2, (height - SIDE) // 2)]
    for fx, fy in ((0.15, 0.2), (0.7, 0.15), (0.2, 0.75), (0.8, 0.7)):
        out.append((int(fx * (width - SIDE)), int(fy * (height - SIDE))))
    return [(x, y, x + SIDE, y + SIDE) for x, y in out]


def check_crops(oracle_lib, wl, img, sample_index, spp):
    o = oracle_lib.OracleTracer()
    o.set_scene(wl.scene)
    for crop in crops(wl.width, wl.height):
        x0, y0, x1, y1 = crop
        ref = o.render(wl.camera, wl.width, wl.height, sample_index, wl.max_bounces, spp, crop=crop)
        a = img[y0:y1, x0:x1]
        b = ref[y0:y1, x0:x1]
        assert np.isfinite(a).all()
        same = float(np.all(a == b, axis=-1).mean())
        rel = float(np.abs(a[..., :3] - b[..., :3]).sum()) / (float(np.abs(b[..., :3]).sum()) + 1e-12)
        assert same >= MIN_IDENTICAL and rel <= MAX_REL_L1, f"crop {crop}: identical={same:.4f} relL1={rel:.2e}"


def test_heavy_geometry_full_frame(oracle_lib, gpu):
    # 1920x1080, 1.0M triangles, 2048x1024 dome; 48M-path waves, 64 traversal
    # and 16 shade blocks per SM, hits unsorted (the benchmark's tuning).
    wl = workloads.heavy_geometry()
    assert (wl.width, wl.height) == (1920, 1080)
    gpu.set_scene(wl.scene)
    gpu.set_tuning(wave_paths=48 << 20, trace_blocks_per_sm=64, shade_blocks_per_sm=16, sort_hits=0)
    try:
        img = gpu.render(wl.camera, wl.width, wl.height, 0, wl.max_bounces, 2).copy()
        # A progressive call on top: 3 more samples in one wave.
        img2 = gpu.render(wl.camera, wl.width, wl.height, 2, wl.max_bounces, 3).copy()
    finally:
        gpu.set_tuning()
    check_crops(oracle_lib, wl, img, 0, 2)
    # The running mean after the second call is the mean over samples 0..4.
    o = oracle_lib.OracleTracer()
    o.set_scene(wl.scene)
    crop = crops(wl.width, wl.height)[0]
    x0, y0, x1, y1 = crop
    ref = o.render(wl.camera, wl.width, wl.height, 0, wl.max_bounces, 5, crop=crop)
    a, b = img2[y0:y1, x0:x1], ref[y0:y1, x0:x1]
    rel = float(np.abs(a[..., :3] - b[..., :3]).sum()) / (float(np.abs(b[..., :3]).sum()) + 1e-12)
    assert rel <= 1e-5, rel  # progressive == batched (path_tracer_tests.cpp:143-150)


def test_spectral_stress_full_frame(oracle_lib, gpu):
    # 1280x720, 200k triangles with cutout leaves, dispersive scattering
    # glass and subsurface; 8M-path waves, 64 / 16 blocks per SM, hits in
    # material order (the benchmark's tuning for this scene).
    wl = workloads.spectral_stress()
    assert (wl.width, wl.height) == (1280, 720)
    gpu.set_scene(wl.scene)
    gpu.set_tuning(wave_paths=8 << 20, trace_blocks_per_sm=64, shade_blocks_per_sm=16, sort_hits=1)
    try:
        img = gpu.render(wl.camera, wl.width, wl.height, 0, wl.max_bounces, 2).copy()
    finally:
        gpu.set_tuning()
    check_crops(oracle_lib, wl, img, 0, 2)


def test_closed_box_full_config(oracle_lib, gpu):
    # 256x256, 16 spp, 8 bounces: the whole config, every pixel.
    wl = workloads.closed_box()
    assert (wl.width, wl.height, wl.spp) == (256, 256, 16)
    o = oracle_lib.OracleTracer()
    o.set_scene(wl.scene)
    ref = o.render(wl.camera, wl.width, wl.height, 0, wl.max_bounces, wl.spp)
    gpu.set_scene(wl.scene)
    img = gpu.render(wl.camera, wl.width, wl.height, 0, wl.max_bounces, wl.spp)
    same = float(np.all(img == ref, axis=-1).mean())
    rel = float(np.abs(img[..., :3] - ref[..., :3]).sum()) / (float(np.abs(ref[..., :3]).sum()) + 1e-12)
    assert same >= MIN_IDENTICAL and rel <= MAX_REL_L1, f"identical={same:.4f} relL1={rel:.2e}"
