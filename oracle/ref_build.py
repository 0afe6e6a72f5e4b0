"""Recipe: compile the reference integrator's own GLSL source as C++ for the CPU.

TEST INFRASTRUCTURE ONLY. Reads the GLSL compute shader held in the raw
strings of src/gpu/vulkan_path_tracer.cpp in the reference checkout, rewrites
the constructs C++ cannot express, and compiles the result with
oracle/ref_glsl_compat.h and oracle/ref_harness.cpp into
oracle/_ref/libhdcx_ref.so. Only oracle/_ref/ receives output (git-ignored).
The reference's C++ host code needs Vulkan, volk and glslang and is not built.

Rewrites (everything else is compiled as written):
  * #version/#extension lines and the local_size layout are dropped;
  * buffer blocks `layout(...) buffer X { T name[]; };` become `static T* name`,
    the CameraBlock uniform a static struct, other uniforms static objects;
  * `inout T x` / `out T x` parameters become `T& x`;
  * unsuffixed floating-point literals get an `f` suffix (GLSL literals are
    binary32);
  * swizzle reads `.rgb .xyz .xy .yz .yzw .rg` become method calls and the one
    swizzle write `mapped.xy *= scale;` is split per component;
  * vector constructors whose arguments call randomFloat more than once are
    brace-initialised, because GLSL evaluates arguments left to right and C++
    function-style calls do not promise an order;
  * main() becomes glsl_main().
"""
from __future__ import annotations

import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
# The hdCodex checkout: $HDCX_REFERENCE_ROOT, else a checkout named
# "reference" beside this repository's root directory.
REFERENCE = os.environ.get("HDCX_REFERENCE_ROOT") or os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference")
SOURCE = os.path.join(REFERENCE, "src", "gpu", "vulkan_path_tracer.cpp")
LIB = os.path.join(OUT, "libhdcx_ref.so")


def extract_glsl(text: str) -> str:
    segments = re.findall(r'R"glsl\((.*?)\)glsl"', text, re.S)
    if not segments:
        raise RuntimeError("no GLSL raw strings found in the reference source")
    return "".join(segments)


def _balanced_end(s: str, open_idx: int) -> int:
    depth = 0
    for i in range(open_idx, len(s)):
        if s[i] == "(":
            depth += 1
        elif s[i] == ")":
            depth -= 1
            if depth == 0:
                return i
    raise ValueError("unbalanced parentheses")


def transform(glsl: str) -> str:
    s = glsl
    s = re.sub(r"^\s*#version.*$", "", s, flags=re.M)
    s = re.sub(r"^\s*#extension.*$", "", s, flags=re.M)
    s = re.sub(r"layout\(local_size[^)]*\)\s*in\s*;", "", s)
    # Buffer blocks with one runtime-sized array member.
    s = re.sub(r"layout\([^)]*\)\s*(?:readonly\s+)?buffer\s+\w+\s*\{\s*(\w+)\s+(\w+)\[\];\s*\}\s*;",
               r"static \1* \2 = nullptr;", s)
    # The camera uniform block.
    s = re.sub(r"layout\([^)]*\)\s*uniform\s+CameraBlock\s*\{(.*?)\}\s*camera\s*;",
               r"static struct CameraBlock {\1} camera;", s, flags=re.S)
    # Remaining uniforms (acceleration structure, sampler array).
    s = re.sub(r"layout\([^)]*\)\s*uniform\s+(\w+)\s+(\w+)(\[\d+\])?\s*;", r"static \1 \2\3;", s)
    if "layout(" in s:
        raise RuntimeError("unhandled layout declaration")
    # Parameter qualifiers.
    s = re.sub(r"\b(?:inout|out)\s+(\w+)\s+(\w+)", r"\1& \2", s)
    # Float literals.
    s = re.sub(r"(?<![\w.])(\d+\.\d*(?:[eE][+-]?\d+)?|\.\d+(?:[eE][+-]?\d+)?|\d+[eE][+-]?\d+)(?![\w.])",
               r"\1f", s)
    # Swizzle write, then swizzle reads.
    s = s.replace("mapped.xy *= scale;", "mapped.x *= scale; mapped.y *= scale;")
    s = re.sub(r"\.(rgb|xyz|yzw|xy|yz|rg)\b(?!\s*\()", r".\1()", s)
    # Constructors with several randomFloat() arguments: brace-initialise.
    out = []
    i = 0
    for m in re.finditer(r"\b(u?vec[234]|ivec2)\(", s):
        start = m.start()
        if start < i:
            continue
        open_idx = m.end() - 1
        end = _balanced_end(s, open_idx)
        body = s[open_idx + 1:end]
        if body.count("randomFloat(") >= 2:
            out.append(s[i:start])
            out.append(f"{m.group(1)}{{{body}}}")
            i = end + 1
    out.append(s[i:])
    s = "".join(out)
    s = re.sub(r"\bvoid\s+main\s*\(\s*\)", "static void glsl_main()", s)
    return s


def build(verbose: bool = False) -> str:
    if not os.path.exists(SOURCE):
        raise FileNotFoundError(f"reference source not found: {SOURCE}")
    os.makedirs(OUT, exist_ok=True)
    with open(SOURCE) as f:
        cpp = transform(extract_glsl(f.read()))
    inc = os.path.join(OUT, "glsl_as_cpp.inc")
    with open(inc, "w") as f:
        f.write("// Generated from the reference's GLSL by oracle/ref_build.py; not committed.\n")
        f.write(cpp)
    srcs = [os.path.join(HERE, n) for n in ("ref_harness.cpp", "oracle_scene.cpp", "oracle_trace.cpp",
                                            "oracle_integrator.cpp")]
    cmd = [os.environ.get("CXX", "g++"), "-std=c++20", "-O2", "-fPIC", "-shared", "-ffp-contract=off",
           "-fno-fast-math", "-w", "-I", os.path.join(os.path.dirname(HERE), "include"), "-I", HERE, "-I", OUT,
           "-o", LIB] + srcs + ["-lpthread"]
    if verbose:
        print(" ".join(cmd))
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"compiling the reference shader failed:\n{res.stderr[-6000:]}")
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
