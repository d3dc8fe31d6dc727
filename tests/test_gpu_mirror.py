"""Builds and runs tests/cpp/mirror_test.cpp: the reference-shaped C++ classes of
include/dgt_mirror.hpp driven like the reference's own test drivers."""
import os
import subprocess

import pytest
from devutil import check_cannon_driver_logs

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


def test_cpp_cannon_drivers_and_logs(tmp_path):
    """include/dgt_drivers.hpp: fullOffloadSumma25Dgemm / preDistributedSumma25Dgemm results
    against host triple loops (tests/cpp/driver_test.cpp), then their CSV rows read back
    the way the thesis notebooks read them."""
    lib = os.path.join(ROOT, "distributed-gemm-thesis_b200", "lib")
    exe = str(tmp_path / "driver_test")
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    subprocess.run(["g++", "-std=c++17", "-O2", os.path.join(ROOT, "tests", "cpp", "driver_test.cpp"),
                    "-I", os.path.join(ROOT, "include"), "-I", os.path.join(cuda, "include"), "-L", lib, "-ldgt",
                    "-L", os.path.join(cuda, "lib64"), "-lcudart", f"-Wl,-rpath,{lib}", "-o", exe], check=True)
    logs = tmp_path / "logs"
    logs.mkdir()
    out = subprocess.run([exe, str(logs)], capture_output=True, text=True, timeout=300)
    print(out.stdout)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "ALL OK" in out.stdout

    check_cannon_driver_logs(logs)
