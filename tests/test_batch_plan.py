"""The batch's lane plan (hdcodex_b200/csrc/batch_plan.h): every job in exactly
one lane, largest first onto the lightest lane, lane waves bounded by the
largest job, the maximum wave and the budget share. Host-only C++, compiled
and run here with g++ (tests/cpp/batch_plan_tests.cpp)."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_lane_plan_rules(tmp_path):
    exe = tmp_path / "batch_plan_tests"
    src = os.path.join(ROOT, "tests", "cpp", "batch_plan_tests.cpp")
    build = subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror",
                            "-I", os.path.join(ROOT, "hdcodex_b200", "csrc"), src, "-o", str(exe)],
                           capture_output=True, text=True)
    assert build.returncode == 0, build.stderr
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert run.returncode == 0, run.stdout + run.stderr
    assert "all batch plan checks passed" in run.stdout
