"""The C++ drop-in shim (include/hdcx/cuda_path_tracer.h).

* It compiles and links against libhdcx.so with this repository's scene types
  and, where the reference checkout exists, against the reference's own
  include/hdcodex/core/versioned_scene.h (HDCX_USE_EXTERNAL_SCENE_ABI), which
  is what a Hydra delegate does.
* On a B200, tests/cpp/path_tracer_tests.cpp (the reference's GPU test
  flow through CudaPathTracer) runs and passes.
"""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BUILD = os.path.join(ROOT, "hdcodex_b200", "_build")
LIBDIR = os.path.join(ROOT, "hdcodex_b200")


def compile_test(hdcx_lib, extra=None, source=None, out="cpp_path_tracer_tests"):
    os.makedirs(BUILD, exist_ok=True)
    exe = os.path.join(BUILD, out)
    src = source or os.path.join(ROOT, "tests", "cpp", "path_tracer_tests.cpp")
    cmd = ["g++", "-std=c++20", "-O1", "-I", os.path.join(ROOT, "include"), src, "-L", LIBDIR, "-lhdcx",
           f"-Wl,-rpath,{LIBDIR}", "-o", exe] + (extra or [])
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
    return exe


def test_shim_compiles_and_links(hdcx_lib):
    exe = compile_test(hdcx_lib)
    assert os.path.exists(exe)


def test_shim_compiles_against_reference_scene_abi(hdcx_lib, tmp_path):
    import ref_build
    ref_include = os.path.join(ref_build.REFERENCE, "include")
    if not os.path.isdir(ref_include):
        pytest.skip("the reference checkout is not present")
    src = tmp_path / "with_reference_abi.cpp"
    src.write_text(
        '#define HDCX_USE_EXTERNAL_SCENE_ABI\n'
        '#include "hdcodex/core/versioned_scene.h"\n'
        '#include "hdcodex/gpu/vulkan_path_tracer.h"\n'
        '#include "hdcx/cuda_path_tracer.h"\n'
        'int main() {\n'
        '  hdcodex::VersionedScene scene;\n'
        '  hdcodex::SceneMesh mesh; mesh.id = "/m"; scene.UpsertMesh(mesh); (void)scene.Publish();\n'
        '  if (!hdcodex::IsCudaPathTracingSupported()) return 0;\n'
        '  hdcodex::CudaPathTracer tracer(0);\n'
        '  tracer.SetScene(scene.Snapshot());\n'
        '  hdcodex::PathTracerCamera camera{};\n'
        '  return tracer.Render(camera, 4, 4, 0).empty() ? 0 : 1;\n'
        '}\n')
    # Only the reference's header-only scene ABI is used; nothing of it is copied.
    compile_test(hdcx_lib, extra=["-I", ref_include, "-fsyntax-only"], source=str(src), out="ref_abi_check")


def test_shim_without_gpu_reports_no_device(hdcx_lib):
    supported, _ = hdcx_lib.probe_devices()
    if supported:
        pytest.skip("an sm_100 device is present")
    exe = compile_test(hdcx_lib)
    res = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert res.returncode == 2, res.stdout


@pytest.mark.gpu
def test_reference_flow_through_cuda_path_tracer(hdcx_lib):
    exe = compile_test(hdcx_lib)
    res = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    assert res.returncode == 0, res.stdout + res.stderr
    assert "passed" in res.stdout
