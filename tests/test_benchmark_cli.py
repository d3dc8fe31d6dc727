"""The 2.5D Cannon benchmark command line (distributed-gemm-thesis_b200/apps/
cublas25d_benchmark.cpp), which keeps the reference's arguments
(src/Benchmarks/cuBLAS25Benchmark.cpp:12-40), linked here against the host-memory test
double of the CUDA runtime and libdgt (tests/cpp/fake_device.cpp): the pre-distributed and
full-offload runs append the reference's CSV rows, and bad arguments end with a message and
a non-zero status instead of an MPI abort."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


@pytest.fixture(scope="module")
def cli(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("cli") / "bench_fake")
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Werror",
                    os.path.join(ROOT, "distributed-gemm-thesis_b200", "apps", "cublas25d_benchmark.cpp"),
                    os.path.join(ROOT, "tests", "cpp", "fake_device.cpp"), "-I", os.path.join(ROOT, "include"),
                    "-I", os.path.join(CUDA, "include"), "-o", exe], check=True)
    return lambda *args: subprocess.run([exe, *map(str, args)], capture_output=True, text=True, timeout=120)


def test_pre_distributed_and_full_offload_rows(cli, tmp_path):
    pd = pytest.importorskip("pandas")
    r = cli("NN", 64, 64, 64, 1.0, 0.0, 2, 2, 1, 2, "devices", "--machine", "b200test", "--logdir", tmp_path)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "Running Pre Distributed" in r.stdout
    r = cli("NN", 96, 96, 96, 1.5, -0.5, 4, 4, 2, 1, "host", 1, "--machine", "b200test", "--logdir", tmp_path,
            "--mode", "ozaki2")
    assert r.returncode == 0, r.stdout + r.stderr
    assert "Running Full Offload" in r.stdout
    pre = pd.read_csv(tmp_path / "DGEMM_execution_logs-PreDistributed_GEMM-b200test-2.5DCANNON-dgt.csv", header=0)
    full = pd.read_csv(tmp_path / "DGEMM_execution_logs-FullOffload_GEMM-b200test-2.5DCANNON-dgt.csv", header=0)
    assert list(pre["M"]) == [64, 64] and list(pre["StackSize"]) == [1, 1]
    assert list(full["Algo"]) == ["2.5D CANNON dgt OzakiII-15moduli"] and list(full["dRow"]) == [4]
    assert (pre["GFlops"] > 0).all() and (full["GFlops"] > 0).all()


def test_bad_arguments(cli, tmp_path):
    assert cli("NN", 64, 64).returncode == 1  # too few arguments: usage
    r = cli("NN", 64, 64, 64, 1.0, 0.0, 2, 2, 1, 1, "cloud")
    assert r.returncode == 2 and "not recognized" in r.stdout
    r = cli("NN", 64, 64, 32, 1.0, 0.0, 2, 2, 1, 1, "devices", "--logdir", tmp_path)
    assert r.returncode == 3 and "M = N = K" in r.stderr  # the reference's constructor rule
    assert cli("NN", 64, 64, 64, 1.0, 0.0, 2, 2, 1, 1, "devices", "--mode", "fp128").returncode == 1
