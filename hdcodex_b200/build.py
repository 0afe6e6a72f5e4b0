"""Builds libhdcx.so, the sm_100a CUDA library behind include/hdcx.h.

Every translation unit is compiled by nvcc for sm_100a only
(-gencode arch=compute_100a,code=sm_100a) with -fmad=false, so that every
float operation is one IEEE operation as the integrator's arithmetic contract
requires; host code is compiled with -ffp-contract=off for the same reason.
Objects go to hdcodex_b200/_build/, the library to hdcodex_b200/libhdcx.so.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libhdcx.so")
INCLUDE = os.path.join(ROOT, "include")

SOURCES = [
    "bvh_build.cu",
    "integrator.cu",
    "nrc.cu",
    "render_static.cu",
    "scene_pack.cpp",
    "device_memory.cpp",
    "hdcx_api.cpp",
]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the hdcx library needs the CUDA 12.9 toolkit")


def cuda_include() -> str:
    return os.path.join(os.path.dirname(os.path.dirname(nvcc())), "include")


def _command(src: str, path: str, obj: str):
    if src.endswith(".cu"):
        return [nvcc()] + ARCH + ["-std=c++17", "-O3", "-lineinfo", "-fmad=false", "-I", INCLUDE, "-I", CSRC,
                                  "-Xcompiler", "-fPIC,-ffp-contract=off,-fvisibility=hidden",
                                  "--expt-relaxed-constexpr", "-Xptxas", "-warn-spills", "-c", path, "-o", obj]
    # Host C++: the reference's host packing arithmetic, IEEE without contraction.
    return [os.environ.get("CXX", "g++"), "-std=c++20", "-O2", "-fPIC", "-ffp-contract=off", "-fno-fast-math",
            "-fvisibility=hidden", "-Wall", "-I", INCLUDE, "-I", CSRC, "-I", cuda_include(), "-c", path, "-o", obj]


def _compile(src: str, verbose: bool) -> str:
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    path = os.path.join(CSRC, src)
    deps = [path] + [os.path.join(CSRC, d) for d in os.listdir(CSRC) if d.endswith((".h", ".cuh"))]
    deps += [os.path.join(CSRC, "device", d) for d in os.listdir(os.path.join(CSRC, "device"))]
    deps.append(os.path.join(INCLUDE, "hdcx.h"))
    hdr_dir = os.path.join(INCLUDE, "hdcx")
    if os.path.isdir(hdr_dir):
        deps += [os.path.join(hdr_dir, d) for d in os.listdir(hdr_dir)]
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(d) for d in deps):
        return obj
    cmd = _command(src, path, obj)
    if verbose:
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{res.stdout}\n{res.stderr}")
    if verbose and res.stderr.strip():
        print(res.stderr, flush=True)
    return obj


def build(verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=min(8, len(SOURCES))) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), SOURCES))
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objs + ["-lpthread", "-ldl"]
        if verbose:
            print(" ".join(cmd), flush=True)
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
