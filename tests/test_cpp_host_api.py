"""The C++ host mirror of the plan API (include/pencil_b200.hpp), compiled
and run as a separate program linked against the library: geometry and
preflight errors without a GPU; plans, a transpose pair and in-place arrays
on the GPU."""

import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "pencil-rs_b200", "pencil_b200")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


@pytest.fixture(scope="module")
def program(tmp_path_factory):
    if shutil.which("g++") is None or not os.path.exists(os.path.join(LIBDIR, "libpencil_b200.so")):
        pytest.skip("needs g++ and the built library")
    exe = str(tmp_path_factory.mktemp("cpp") / "host_api")
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-I", os.path.join(ROOT, "include"), "-I",
           os.path.join(CUDA, "include"), os.path.join(ROOT, "tests", "cpp", "host_api.cpp"), "-o", exe,
           "-L", LIBDIR, "-lpencil_b200", "-Wl,-rpath," + LIBDIR, "-L", os.path.join(CUDA, "lib64"),
           "-lcudart", "-Wl,-rpath," + os.path.join(CUDA, "lib64")]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    assert proc.returncode == 0, proc.stderr
    return exe


def test_cpp_mirror_host_geometry_and_preflight(program):
    proc = subprocess.run([program, "host"], capture_output=True, text=True, timeout=60)
    assert proc.returncode == 0 and "host ok" in proc.stdout, proc.stdout + proc.stderr


@pytest.mark.gpu
def test_cpp_mirror_on_the_gpu(program):
    proc = subprocess.run([program, "gpu"], capture_output=True, text=True, timeout=300)
    assert proc.returncode == 0 and "gpu ok" in proc.stdout, proc.stdout + proc.stderr
