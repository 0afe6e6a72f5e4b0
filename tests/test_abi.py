"""The C ABI library: loads, exports every declared entry point, struct layouts
agree with the Python mirrors, defaults agree with the reference's scene ABI.
No compute call needs a GPU here."""
import ctypes as C
import os
import re

import pytest

from hdcodex_b200 import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "hdcx.h")).read()
    return sorted(set(re.findall(r"HDCX_API\s+[\w\s\*]+?\b(hdcx_\w+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared_symbols()
    assert "hdcx_render" in names and "hdcx_set_scene" in names and "hdcx_create" in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol(hdcx_lib):
    lib = hdcx_lib.lib()
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, f"libhdcx.so does not export {missing}"


def test_python_binding_covers_every_symbol(hdcx_lib):
    from hdcodex_b200.tracer import SIGNATURES
    assert sorted(SIGNATURES) == declared_symbols()


def test_struct_sizes_match_ctypes(hdcx_lib):
    lib = hdcx_lib.lib()
    sizes = (C.c_uint64 * 16)()
    n = lib.hdcx_abi_struct_sizes(sizes, 16)
    assert n == len(_abi.STRUCTS_IN_ABI_ORDER)
    for i, struct in enumerate(_abi.STRUCTS_IN_ABI_ORDER):
        assert sizes[i] == C.sizeof(struct), struct.__name__
    assert lib.hdcx_abi_version() == 1


def test_material_and_light_defaults_match(hdcx_lib):
    lib = hdcx_lib.lib()
    m = _abi.MaterialDesc()
    lib.hdcx_material_defaults(C.byref(m))
    for name, ctype, default in _abi.MATERIAL_FIELDS:
        value = getattr(m, name)
        if ctype is C.c_char_p:
            assert value is None
        elif ctype is _abi.F3:
            assert list(value) == pytest.approx(list(default)), name
        else:
            assert value == pytest.approx(float(default)), name
    l = _abi.LightDesc()
    lib.hdcx_light_defaults(C.byref(l))
    for name, ctype, default in _abi.LIGHT_FIELDS:
        value = getattr(l, name)
        if ctype is C.c_char_p:
            assert value is None
        elif ctype is _abi.F3:
            assert list(value) == pytest.approx(list(default)), name
        else:
            assert value == pytest.approx(float(default)), name


def test_probe_and_create_fail_cleanly_without_sm100(hdcx_lib):
    supported, count = hdcx_lib.probe_devices()
    if supported:
        pytest.skip("an sm_100 device is present")
    handle = C.c_void_p()
    status = hdcx_lib.lib().hdcx_create(0, C.byref(handle))
    assert status in (4, 5)  # NO_DEVICE or UNSUPPORTED: there is no CPU fallback
    with pytest.raises(RuntimeError):
        hdcx_lib.PathTracer()


def test_raster_preview_is_rejected_without_a_device(hdcx_lib):
    # The C++ shim and the Python binding both reject RasterPreview before any
    # device call (vulkan_path_tracer.cpp:2495-2498 throws invalid_argument).
    tracer = object.__new__(hdcx_lib.PathTracer)
    tracer._h = None
    with pytest.raises(ValueError):
        hdcx_lib.PathTracer.set_shading_mode(tracer, hdcx_lib.RASTER_PREVIEW)


C_STRUCT_NAMES = ["hdcx_camera", "hdcx_mesh_desc", "hdcx_material_desc", "hdcx_texture_desc", "hdcx_light_desc",
                  "hdcx_scene_desc", "hdcx_packed_texture", "hdcx_packed_scene", "hdcx_render_stats",
                  "hdcx_batch_job", "hdcx_nrc_config", "hdcx_tuning", "hdcx_instancer_desc", "hdcx_scene_info"]


def test_struct_fields_match_the_header(tmp_path):
    """Every field of every Python mirror has the header's name and offset:
    gcc compiles offsetof() of each field against include/hdcx.h."""
    import subprocess
    assert len(C_STRUCT_NAMES) == len(_abi.STRUCTS_IN_ABI_ORDER)
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "hdcx.h"', "int main(void) {"]
    expected = []
    for cname, struct in zip(C_STRUCT_NAMES, _abi.STRUCTS_IN_ABI_ORDER):
        for field, _ctype in struct._fields_:
            lines.append(f'  printf("%zu\\n", offsetof({cname}, {field}));')
            expected.append((cname, field, getattr(struct, field).offset))
        lines.append(f'  printf("%zu\\n", sizeof({cname}));')
        expected.append((cname, "sizeof", C.sizeof(struct)))
    lines.append("  return 0;\n}")
    src = tmp_path / "offsets.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "offsets"
    build = subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                           capture_output=True, text=True)
    assert build.returncode == 0, build.stderr
    got = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    assert len(got) == len(expected)
    mismatched = [(c, f, e, g) for (c, f, e), g in zip(expected, got) if e != g]
    assert not mismatched, mismatched


def test_device_memory_budget_entry_points(hdcx_lib):
    """The budget is host bookkeeping: settable and readable without a GPU,
    device ordinals outside 0..63 are rejected."""
    from hdcodex_b200.tracer import device_memory_usage, set_device_memory_limit
    set_device_memory_limit(5, 123456)
    used, limit = device_memory_usage(5)
    assert limit == 123456 and used == 0
    set_device_memory_limit(5, 0)
    assert device_memory_usage(5) == (0, 0)
    with pytest.raises(RuntimeError):
        set_device_memory_limit(64, 1)
    with pytest.raises(RuntimeError):
        set_device_memory_limit(-1, 1)
