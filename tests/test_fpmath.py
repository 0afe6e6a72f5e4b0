"""The binary32 transcendental functions of include/hdcx/fpmath.h.

The integrator evaluates exp, log, pow, sin, cos, acos and atan2 with these
functions on the GPU, and the oracle and the reference-shader harness evaluate
them with the same functions on the CPU; bit-exact parity of the renders rests
on the two evaluations agreeing.

* CPU: accuracy against binary64 libm over the integrator's argument ranges
  (tests/cpp/fpmath_accuracy.cpp states the per-function ulp bounds), special
  values, and that the header also compiles as C.
* GPU: device results equal host results bit for bit on 4M arguments, ordinary
  ranges plus arbitrary bit patterns (tests/cuda/fpmath_device.cu).
"""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(ROOT, "hdcodex_b200", "_build")


def _compile(cmd):
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr


def _parse(stdout):
    rows = {}
    for line in stdout.splitlines():
        parts = line.split()
        if len(parts) >= 3 and not line.startswith(" "):
            rows[parts[0]] = parts[1:]
    return rows


def test_accuracy_against_binary64():
    os.makedirs(BUILD, exist_ok=True)
    exe = os.path.join(BUILD, "fpmath_accuracy")
    _compile(["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-fno-fast-math", "-I", INCLUDE,
              os.path.join(ROOT, "tests", "cpp", "fpmath_accuracy.cpp"), "-o", exe])
    res = subprocess.run([exe, "1000000"], capture_output=True, text=True, timeout=300)
    rows = _parse(res.stdout)
    assert res.returncode == 0, res.stdout
    for name in ("sin", "cos", "exp", "log", "acos", "atan2", "pow", "pow5"):
        samples, max_ulp, violations = rows[name]
        assert int(samples) > 100000
        assert int(violations) == 0, (name, max_ulp)
    assert rows["pow5"][1] == "0.0"  # x^5 through exact binary64 products rounds once


def test_header_compiles_as_c(tmp_path):
    src = tmp_path / "fpmath_c.c"
    src.write_text('#include "hdcx/fpmath.h"\n'
                   'float f(float x) { return hdcx_fp_pow(hdcx_fp_sin(x), 2.5f) + hdcx_fp_atan2(x, 1.0f); }\n')
    _compile(["gcc", "-std=c99", "-Wall", "-Werror", "-fsyntax-only", "-I", INCLUDE, str(src)])


@pytest.mark.gpu
def test_device_matches_host_bit_for_bit():
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    os.makedirs(BUILD, exist_ok=True)
    exe = os.path.join(BUILD, "fpmath_device")
    _compile([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "-O2", "-fmad=false",
              "-Xcompiler", "-ffp-contract=off", "-I", INCLUDE,
              os.path.join(ROOT, "tests", "cuda", "fpmath_device.cu"), "-o", exe])
    res = subprocess.run([exe, str(1 << 22)], capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stdout + res.stderr
    rows = _parse(res.stdout)
    for name in ("sin", "cos", "exp", "log", "pow", "pow5", "acos", "atan2"):
        assert rows[name][1] == "0", res.stdout
