"""The render views beyond the reference's Render call: the GPU interactive
preview, the asynchronous double-buffered read-back and the primary-hit AOVs.

* hdcx_render_preview follows HdCodexRenderPass::_Execute's interactive branch
  (render_pass.cpp:191-208): a render at ceil(w/2) x ceil(h/2), sample 0, two
  bounces, one sample, upscaled by the reference's UpscaleNearest rule
  (render_pass.cpp:45-68, restated here in numpy). It must equal that render
  of the oracle, upscaled the same way, at the parity tolerance.
* hdcx_render_async / hdcx_wait_render give the same images as hdcx_render
  for the same calls, with two frames in flight.
* With hdcx_set_aovs every render writes the primary hit of its first sample:
  equal to hdcx_trace_primary and to the oracle's primary hits, bit for bit.
"""
import numpy as np
import pytest

import ref_scenes as R
from hdcodex_b200 import PathTracer, workloads

pytestmark = pytest.mark.gpu

MIN_IDENTICAL = 0.99
MAX_REL_L1 = 1e-3


def upscale_nearest(src, width, height):
    """render_pass.cpp:45-68 in numpy: source = min(size - 1, dest * size // dest_size)."""
    sh, sw = src.shape[:2]
    ys = np.minimum(sh - 1, (np.arange(height, dtype=np.int64) * sh) // height)
    xs = np.minimum(sw - 1, (np.arange(width, dtype=np.int64) * sw) // width)
    return src[ys][:, xs]


def close(img, ref):
    same = float(np.all(img == ref, axis=-1).mean())
    rel = float(np.abs(img[..., :3] - ref[..., :3]).sum()) / (float(np.abs(ref[..., :3]).sum()) + 1e-12)
    return same >= MIN_IDENTICAL and rel <= MAX_REL_L1, (same, rel)


@pytest.mark.parametrize("size", [(64, 64), (65, 33), (1, 1), (97, 40)])
def test_preview_is_the_half_resolution_render_upscaled(oracle_lib, size):
    w, h = size
    wl = workloads.closed_box(width=w, height=h)
    tw, th = max(1, (w + 1) // 2), max(1, (h + 1) // 2)
    o = oracle_lib.OracleTracer()
    o.set_scene(wl.scene)
    ref = upscale_nearest(o.render(wl.camera, tw, th, 0, 2, 1), w, h)
    with PathTracer(0) as t:
        t.set_scene(wl.scene)
        img = t.render_preview(wl.camera, w, h)
        assert img.shape == (h, w, 4)
        ok, info = close(img, ref)
        assert ok, info
        # The same as the tracer's own half-resolution render, upscaled.
        half = t.render(wl.camera, tw, th, 0, 2, 1)
        assert np.array_equal(img, upscale_nearest(half, w, h))


def test_preview_without_geometry_writes_nothing():
    with PathTracer(0) as t:
        assert t.render_preview(R.base_camera(), 16, 16) is None


def test_async_frames_equal_sync_renders():
    wl = workloads.closed_box(width=48, height=40)
    calls = [(0, 2), (2, 3), (5, 1), (0, 2), (2, 1)]
    with PathTracer(0) as sync:
        sync.set_scene(wl.scene)
        expected = [sync.render(wl.camera, 48, 40, si, 8, sc).copy() for si, sc in calls]
    with PathTracer(0) as t:
        t.set_scene(wl.scene)
        tickets = []
        images = {}
        for k, (si, sc) in enumerate(calls):
            tickets.append(t.render_async(wl.camera, 48, 40, si, 8, sc))
            if k >= 1:  # two frames in flight; collect the older one
                images[k - 1] = t.wait_render(tickets[k - 1], 48, 40)
        images[len(calls) - 1] = t.wait_render(tickets[-1], 48, 40)
        assert tickets == list(range(len(calls)))
        for k, img in images.items():
            assert np.array_equal(img, expected[k]), k
        # The image of a ticket two calls back is no longer held.
        with pytest.raises(RuntimeError, match="not held"):
            t.wait_render(tickets[0], 48, 40)
        # A synchronous render after async frames continues the running mean.
        img = t.render(wl.camera, 48, 40, 3, 8, 1)
        assert np.isfinite(img).all()


def test_async_waiting_out_of_order_completes_in_order():
    wl = workloads.closed_box(width=32, height=32)
    with PathTracer(0) as sync:
        sync.set_scene(wl.scene)
        a = sync.render(wl.camera, 32, 32, 0, 8, 1).copy()
        b = sync.render(wl.camera, 32, 32, 1, 8, 2).copy()
    with PathTracer(0) as t:
        t.set_scene(wl.scene)
        t0 = t.render_async(wl.camera, 32, 32, 0, 8, 1)
        t1 = t.render_async(wl.camera, 32, 32, 1, 8, 2)
        got_b = t.wait_render(t1, 32, 32)
        got_a = t.wait_render(t0, 32, 32)
        assert np.array_equal(got_a, a) and np.array_equal(got_b, b)
        assert t.stats()["spectral_paths"] == 32 * 32 * 3 * 2


def test_aovs_are_the_primary_hits_of_the_first_sample(oracle_lib):
    wl = workloads.heavy_geometry(width=160, height=90, spp=2, dome_size=(64, 32))
    o = oracle_lib.OracleTracer()
    o.set_scene(wl.scene)
    with PathTracer(0) as t:
        t.set_scene(wl.scene)
        t.set_aovs(3)
        for sample_index in (0, 2):
            t.render(wl.camera, wl.width, wl.height, sample_index, 8, 2)
            ids, depth = t.read_aovs(wl.width, wl.height)
            p, d = t.trace_primary(wl.camera, wl.width, wl.height, sample_index)
            rp, rd = o.trace_primary(wl.camera, wl.width, wl.height, sample_index)
            assert np.array_equal(ids, p) and np.array_equal(depth.view(np.uint32), d.view(np.uint32))
            assert np.array_equal(ids, rp) and np.array_equal(depth.view(np.uint32), rd.view(np.uint32))
            assert (ids != 0xFFFFFFFF).mean() > 0.3
        t.set_aovs(0)
        with pytest.raises(RuntimeError):
            t.set_aovs(4)
