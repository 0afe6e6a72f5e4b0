"""hdcx_render_static, the render entry point that allocates no device memory,
against hdcx_render on the same scene, camera and calls.

The file name makes pytest collect it last, so that it runs after every other
GPU test has used the library in this process; it also passes alone in a
fresh process. Each case makes two calls in a row (a first render, then a
progressive one that reads the running mean back), because every call shares
the library's one static scratch array and it keeps the last call's contents.
The tolerance is the one the GPU parity tests use.
"""
import ctypes as C

import numpy as np
import pytest

import ref_scenes as R
from hdcodex_b200 import PathTracer, workloads

pytestmark = pytest.mark.gpu

MIN_IDENTICAL = 0.99
MAX_REL_L1 = 1e-3
MAX_PIXELS = 1 << 20
INVALID_ARGUMENT = 1


def compare(img, ref):
    same = np.all(img == ref, axis=-1)
    denom = float(np.abs(ref[..., :3]).sum()) + 1e-12
    return float(same.mean()), float(np.abs(img[..., :3] - ref[..., :3]).sum()) / denom


def render_static(tracer, camera, w, h, sample_index, bounces, spp, device_ptr):
    from hdcodex_b200.tracer import lib
    written = C.c_int32(0)
    status = lib().hdcx_render_static(tracer.handle, C.byref(camera), w, h, sample_index, bounces, spp,
                                      C.c_void_p(device_ptr), C.byref(written))
    return status, written.value


CASES = {
    # 64x64: a frame's paths fit one wave several samples at a time.
    "base_64x64": (R.base_scene, R.base_camera, 64, 64),
    # 320x240: more than one wave per sample (the wave is 65,536 paths).
    "closed_box_320x240": (lambda: workloads.closed_box(320, 240).scene,
                           lambda: workloads.closed_box(320, 240).camera, 320, 240),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_static_render_matches_render_two_calls(hdcx_lib, case):
    import torch
    make_scene, make_camera, w, h = CASES[case]
    camera = make_camera()
    device_image = torch.zeros((h, w, 4), dtype=torch.float32, device="cuda:0")
    with PathTracer(0) as tracer:
        tracer.set_scene(make_scene())
        for sample_index, spp in ((0, 3), (3, 2)):
            ref = tracer.render(camera, w, h, sample_index, 8, spp)
            torch.cuda.synchronize()
            status, written = render_static(tracer, camera, w, h, sample_index, 8, spp, device_image.data_ptr())
            assert status == 0, tracer_error(tracer)
            assert written == 1
            img = device_image.cpu().numpy()
            assert np.isfinite(img).all()
            frac, rel = compare(img, ref)
            assert frac >= MIN_IDENTICAL and rel <= MAX_REL_L1, (case, sample_index, frac, rel)


def test_static_render_allocates_no_device_memory(hdcx_lib):
    """The property the entry point exists for: after the first call on the
    device (which looks up the static array's address and loads the kernels),
    further calls leave the device's free memory unchanged, including a call
    at a new, larger image size, where hdcx_render would grow its buffers."""
    import torch
    camera = R.base_camera()
    small = torch.zeros((48, 48, 4), dtype=torch.float32, device="cuda:0")
    large = torch.zeros((300, 400, 4), dtype=torch.float32, device="cuda:0")
    with PathTracer(0) as tracer:
        tracer.set_scene(R.base_scene())
        status, _ = render_static(tracer, camera, 48, 48, 0, 8, 1, small.data_ptr())
        assert status == 0, tracer_error(tracer)
        torch.cuda.synchronize()
        free_before, _ = torch.cuda.mem_get_info(0)
        for w, h, image in ((48, 48, small), (400, 300, large), (48, 48, small)):
            for sample_index, spp in ((0, 2), (2, 1)):
                status, written = render_static(tracer, camera, w, h, sample_index, 8, spp, image.data_ptr())
                assert status == 0 and written == 1, tracer_error(tracer)
        torch.cuda.synchronize()
        free_after, _ = torch.cuda.mem_get_info(0)
        assert free_after == free_before, (free_before, free_after)
        assert torch.isfinite(large).all().item()


def test_static_render_restart_ignores_buffer_contents(hdcx_lib):
    """sample_index 0 does not read the caller's buffer: NaN left in it (a
    recycled or uninitialised allocation) does not reach the image."""
    import torch
    camera = R.base_camera()
    with PathTracer(0) as tracer:
        tracer.set_scene(R.base_scene())
        ref = tracer.render(camera, 32, 32, 0, 8, 2).copy()
        torch.cuda.synchronize()
        image = torch.full((32, 32, 4), float("nan"), dtype=torch.float32, device="cuda:0")
        status, written = render_static(tracer, camera, 32, 32, 0, 8, 2, image.data_ptr())
        assert status == 0 and written == 1, tracer_error(tracer)
        img = image.cpu().numpy()
        assert np.isfinite(img).all()
        frac, rel = compare(img, ref)
        assert frac >= MIN_IDENTICAL and rel <= MAX_REL_L1, (frac, rel)


def test_static_render_rejects_a_tracer_with_a_radiance_cache(hdcx_lib):
    """The static render has no cache mode; a tracer with a cache attached is
    refused with a message instead of silently rendering plain paths."""
    import torch
    from hdcodex_b200 import RadianceCache
    image = torch.zeros((16, 16, 4), dtype=torch.float32, device="cuda:0")
    with PathTracer(0) as tracer, RadianceCache(0, log2_table_size=12) as cache:
        tracer.set_scene(R.base_scene())
        tracer.set_radiance_cache(cache)
        status, written = render_static(tracer, R.base_camera(), 16, 16, 0, 8, 1, image.data_ptr())
        assert status == INVALID_ARGUMENT and written == 0
        assert "radiance cache" in tracer_error(tracer)
        tracer.set_radiance_cache(None)
        status, written = render_static(tracer, R.base_camera(), 16, 16, 0, 8, 1, image.data_ptr())
        assert status == 0 and written == 1, tracer_error(tracer)


def test_static_render_rejects_images_above_its_maximum(hdcx_lib):
    import torch
    device_image = torch.zeros((4,), dtype=torch.float32, device="cuda:0")
    with PathTracer(0) as tracer:
        tracer.set_scene(R.base_scene())
        status, written = render_static(tracer, R.base_camera(), 1025, 1024, 0, 8, 1, device_image.data_ptr())
        assert status == INVALID_ARGUMENT and written == 0
        assert "exceeds its maximum of 1048576 pixels" in tracer_error(tracer)
        # The largest accepted image renders.
        big = torch.zeros((1024, 1024, 4), dtype=torch.float32, device="cuda:0")
        status, written = render_static(tracer, R.base_camera(), 1024, 1024, 0, 2, 1, big.data_ptr())
        assert status == 0 and written == 1, tracer_error(tracer)
        assert torch.isfinite(big).all().item()


def tracer_error(tracer):
    from hdcodex_b200.tracer import lib
    msg = lib().hdcx_last_error(tracer.handle)
    return msg.decode() if msg else ""
