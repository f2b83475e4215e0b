"""A C++ program bound to the C ABI the way abacus would bind it (no Python
in between): tests/cpp/driver_plan.cpp builds a small box as abacus lays it
out, drives the NearFieldDriver mirror in planner-only mode and checks the
planned DirectTotal for one z-domain and for the nodes of a 2D z-split
against the 5x5x5 pair count.  Built into the package's ignored build
folder; needs no GPU."""
import os
import pathlib
import shutil
import subprocess
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]


def test_cpp_consumer_plans_the_box(capi):
    if shutil.which("g++") is None:
        pytest.skip("g++ not found")
    sys.path.insert(0, str(ROOT / "abacus-public_b200"))
    import build
    cuda_lib = pathlib.Path(build.nvcc()).resolve().parent.parent / "lib64"
    libdir = capi.LIB_PATH.parent
    out_dir = ROOT / "abacus-public_b200" / "_build"
    out_dir.mkdir(exist_ok=True)
    exe = out_dir / "driver_plan"
    r = subprocess.run(["g++", "-pipe", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror",
                        f"-I{ROOT / 'include'}", str(ROOT / "tests" / "cpp" / "driver_plan.cpp"),
                        f"-L{libdir}", "-lnfb200", f"-Wl,-rpath,{libdir}", f"-L{cuda_lib}",
                        f"-Wl,-rpath-link,{cuda_lib}", "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    env = dict(os.environ)
    env["LD_LIBRARY_PATH"] = os.pathsep.join(
        [p for p in (env.get("LD_LIBRARY_PATH", ""), str(cuda_lib)) if p])
    r = subprocess.run([str(exe)], capture_output=True, text=True, env=env, timeout=120)
    assert r.returncode == 0 and r.stdout.startswith("ok "), r.stdout + r.stderr
