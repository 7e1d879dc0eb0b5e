"""A C++ driver in the reference's style, built against include/kbfv_compat.hpp
and libkbfv.so, runs the full encode/encrypt/multiply/decrypt flow on the GPU."""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("cpp") / "compat_mult")
    libdir = os.path.join(ROOT, "kunpbfv_b200")
    nvcc = "/usr/local/cuda/bin/nvcc" if os.path.exists("/usr/local/cuda/bin/nvcc") else "nvcc"
    subprocess.run([nvcc, "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "compat_mult.cpp"), "-L", libdir, "-lkbfv",
                    "-Xlinker", "-rpath", "-Xlinker", libdir, "-o", out], check=True)
    return out


@pytest.mark.parametrize("n", [16384, 32768])
def test_reference_style_driver(driver, n):
    r = subprocess.run([driver, str(n)], capture_output=True, text=True, timeout=600)
    print(r.stdout, r.stderr)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "wrong=0" in r.stdout
