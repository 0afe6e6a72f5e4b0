"""Generates tests/golden/reference_renders.npz from the reference's own shader.

Run where the reference checkout is present (python tests/golden/make_golden.py):
oracle/ref_build.py compiles the GLSL integrator of the reference
(src/gpu/vulkan_path_tracer.cpp) as C++ and this script renders the scenes of
the reference's GPU test (tests/path_tracer_tests.cpp) at 32x32, 4 spp, plus
the 34-triangle closed box at 64x64, 2 spp. The GPU tests compare the CUDA
tracer with these images; the fixture travels with the repository.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")]

import oracle as O  # noqa: E402
import ref_build  # noqa: E402
import ref_scenes as R  # noqa: E402
from hdcodex_b200 import workloads  # noqa: E402

VARIANTS = ["base", "oren_nayar", "udim", "authored_normals", "glossy", "matte_black", "coated", "subsurface",
            "cutout", "opaque_black", "translucent", "thin_walled", "nondispersive", "dispersive", "fallback"]
SIZE = 32
SPP = 4


def main():
    ref_build.build()
    out = {}
    for name in VARIANTS:
        t = O.ReferenceTracer()
        t.set_scene(R.variant(name))
        out[name] = t.render(R.base_camera(), SIZE, SIZE, 0, 8, SPP)
    wl = workloads.closed_box(width=64, height=64)
    t = O.ReferenceTracer()
    t.set_scene(wl.scene)
    out["closed_box"] = t.render(wl.camera, 64, 64, 0, 8, 2)
    np.savez_compressed(os.path.join(HERE, "reference_renders.npz"), **out)
    print("wrote", os.path.join(HERE, "reference_renders.npz"))


if __name__ == "__main__":
    main()
