"""Builds and runs tests/cpp/mirror_test.cpp: the reference-shaped C++ classes of
include/dgt_mirror.hpp driven like the reference's own test drivers."""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_cpp_mirror_classes(tmp_path):
    lib = os.path.join(ROOT, "distributed-gemm-thesis_b200", "lib")
    exe = str(tmp_path / "mirror_test")
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    subprocess.run(["g++", "-std=c++17", "-O2", os.path.join(ROOT, "tests", "cpp", "mirror_test.cpp"),
                    "-I", os.path.join(ROOT, "include"), "-I", os.path.join(cuda, "include"), "-L", lib, "-ldgt",
                    "-L", os.path.join(cuda, "lib64"), "-lcudart", f"-Wl,-rpath,{lib}", "-o", exe], check=True)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    print(out.stdout)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "ALL OK" in out.stdout

