"""The CUDA tracer against images of the reference's own shader.

tests/golden/reference_renders.npz holds renders of the reference's GLSL
integrator compiled as C++ (tests/golden/make_golden.py): the scenes of the
reference's GPU test at 32x32, 4 spp, and the 34-triangle closed box at
64x64, 2 spp. The CUDA tracer must reproduce them bit for bit on at least
99% of pixels (see test_gpu_parity for the tolerance)."""
import os

import numpy as np
import pytest

import ref_scenes as R
from hdcodex_b200 import PathTracer, workloads

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_renders.npz")


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN)


@pytest.fixture(scope="module")
def gpu():
    t = PathTracer(0)
    yield t
    t.close()


@pytest.mark.parametrize("name", ["base", "oren_nayar", "udim", "authored_normals", "glossy", "matte_black",
                                  "coated", "subsurface", "cutout", "opaque_black", "translucent", "thin_walled",
                                  "nondispersive", "dispersive", "fallback"])
def test_reference_variant(gpu, golden, name):
    gpu.set_scene(R.variant(name))
    img = gpu.render(R.base_camera(), 32, 32, 0, 8, 4)
    same = np.all(img == golden[name], axis=-1).mean()
    assert same >= 0.99, f"{name}: {same:.4f} of pixels identical to the reference shader"


def test_closed_box(gpu, golden):
    wl = workloads.closed_box(width=64, height=64)
    gpu.set_scene(wl.scene)
    img = gpu.render(wl.camera, 64, 64, 0, 8, 2)
    assert np.all(img == golden["closed_box"], axis=-1).mean() >= 0.99
