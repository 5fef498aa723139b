"""The reference-signature C++ API (include/tomos/b200.hpp) compiles with
g++ against libtomos_b200.so and passes the C++ mirror of the reference's
LSQR/workspace test cases on the device."""
import os
import subprocess
import tempfile

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def compile_cpp(out):
    cmd = ["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"),
           "-I", "/usr/local/cuda/include", os.path.join(ROOT, "tests", "cpp", "test_api.cpp"),
           "-o", out, "-L", os.path.join(ROOT, "tomos_b200", "lib"), "-ltomos_b200",
           "-L", "/usr/local/cuda/lib64", "-lcudart",
           "-Wl,-rpath," + os.path.join(ROOT, "tomos_b200", "lib"), "-Wl,-rpath,/usr/local/cuda/lib64"]
    subprocess.run(cmd, check=True)


def test_cpp_api_compiles():
    with tempfile.TemporaryDirectory() as d:
        compile_cpp(os.path.join(d, "t"))


@pytest.mark.gpu
def test_cpp_api_runs():
    with tempfile.TemporaryDirectory() as d:
        exe = os.path.join(d, "t")
        compile_cpp(exe)
        r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stdout + r.stderr
        assert "cpp api ok" in r.stdout
