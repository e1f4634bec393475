"""The drop-in boundary builds: the C++ driver written against the facade
(include/gpufem/gpufem.hpp, tests/drivers/linear_static.cpp, shaped like the
reference's examples/plate_demo/linear_static.cu) and the C driver written
against the C ABI (include/gpufem.h, tests/drivers/c_abi_solve.c) compile
and link against libgpufem.so. Nothing runs here (no GPU needed);
tests/test_gpu_boundary.py runs both drivers on a GPU."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
LIB_DIR = os.path.join(ROOT, "gpu_fem_b200")
DRIVERS = os.path.join(ROOT, "tests", "drivers")


def need(tool):
    if shutil.which(tool) is None:
        pytest.skip(f"{tool} not available")
    if not os.path.exists(os.path.join(CUDA, "include", "cuda_runtime.h")):
        pytest.skip("CUDA headers not available")
    if not os.path.exists(os.path.join(LIB_DIR, "libgpufem.so")):
        pytest.skip("libgpufem.so not built")


def build_driver(name, out_dir):
    """Compiles tests/drivers/<name> into out_dir; returns the executable."""
    cpp = name.endswith(".cpp")
    compiler = "g++" if cpp else "gcc"
    need(compiler)
    out = os.path.join(str(out_dir), os.path.splitext(name)[0])
    cmd = [compiler, "-std=c++17" if cpp else "-std=c11", "-O1", "-Wall",
           os.path.join(DRIVERS, name), "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(CUDA, "include"), "-L", LIB_DIR, "-lgpufem",
           "-Wl,-rpath," + LIB_DIR, "-L", os.path.join(CUDA, "lib64"), "-lcudart", "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert "warning" not in r.stderr, r.stderr
    return out


def test_cpp_facade_driver_compiles_and_links(tmp_path):
    build_driver("linear_static.cpp", tmp_path)


def test_c_abi_driver_compiles_and_links(tmp_path):
    build_driver("c_abi_solve.c", tmp_path)
