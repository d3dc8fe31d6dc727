"""CSV execution logs in the reference's schema (include/dgt_logging.hpp), checked on the
CPU: the C++ logger's file names, header placement and row format
(tests/cpp/csv_log_test.cpp), then the file read back the way the thesis notebooks read
it (plotters/executionAnalysis.ipynb: pandas.read_csv(header=0), grouped by Algo, M, N, K,
TotalGPUs, DataLocation; TotalTime = CommunicationTime + GemmCallTime).  The 2.5D Cannon
drivers that write these logs (include/dgt_drivers.hpp) run here against a host-memory test
double of the device layer, are linked against the real library, and run on the GPU in
tests/test_gpu_mirror.py."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INC = os.path.join(ROOT, "include")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
HEADER = ("Algo,M,N,K,TotalNodes,TotalGPUs,dRow,dCol,StackSize,DecompositionTime,ExecutionTime,GatherTime,"
          "GFlops,DataLocation,CommunicationTime,GemmCallTime")


def test_logger_and_notebook_read(tmp_path):
    pd = pytest.importorskip("pandas")
    exe = str(tmp_path / "csv_log_test")
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Werror", os.path.join(ROOT, "tests", "cpp", "csv_log_test.cpp"),
                    "-I", INC, "-o", exe], check=True)
    logs = tmp_path / "logs"
    logs.mkdir()
    out = subprocess.run([exe, str(logs)], capture_output=True, text=True, timeout=60)
    assert out.returncode == 0 and "ALL OK" in out.stdout, out.stdout + out.stderr

    path = logs / "DGEMM_execution_logs-PreDistributed_GEMM-b200-2.5DCANNON-dgt.csv"
    df = pd.read_csv(path, header=0, delimiter=",")
    assert list(df.columns) == HEADER.split(",")
    assert len(df) == 2
    assert list(df["Algo"]) == ["2.5D CANNON dgt", "2.5D CANNON dgt OzakiII-14moduli"]
    assert list(df["StackSize"]) == [2, 1] and list(df["dRow"]) == [4, 2]
    assert (df["DataLocation"] == "devices").all()
    # the notebooks' derived columns and grouping
    df["TotalTime"] = df["CommunicationTime"] + df["GemmCallTime"]
    df["Performance (Tflops)"] = df["GFlops"] / 1024
    g = df.groupby(["Algo", "M", "N", "K", "TotalGPUs", "DataLocation"]).mean(numeric_only=True).reset_index()
    assert len(g) == 2
    assert g.loc[g["M"] == 8192, "GFlops"].iloc[0] == pytest.approx(2 * 8192 ** 3 * 1e-9 / 0.03125, rel=1e-9)


def test_drivers_on_host_test_double(tmp_path):
    """The drivers' host logic (allocation sizes, copy pitches, run loop, result, CSV rows)
    with tests/cpp/fake_device.cpp standing in for the CUDA runtime and libdgt: the same
    program and checks the GPU test runs against the real library."""
    pytest.importorskip("pandas")
    from devutil import check_cannon_driver_logs

    exe = str(tmp_path / "driver_fake")
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror",
                    os.path.join(ROOT, "tests", "cpp", "driver_test.cpp"),
                    os.path.join(ROOT, "tests", "cpp", "fake_device.cpp"),
                    "-I", INC, "-I", os.path.join(CUDA, "include"), "-o", exe], check=True)
    logs = tmp_path / "logs"
    logs.mkdir()
    out = subprocess.run([exe, str(logs)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0 and "ALL OK" in out.stdout, out.stdout + out.stderr
    check_cannon_driver_logs(logs)


def test_drivers_header_compiles_and_links(tmp_path):
    """dgt_drivers.hpp with the CUDA runtime headers, and the GPU driver test linked against
    the library (nothing is run: there may be no GPU)."""
    lib = os.path.join(ROOT, "distributed-gemm-thesis_b200", "lib")
    if not os.path.exists(os.path.join(lib, "libdgt.so")):
        pytest.skip("libdgt.so not built")
    exe = str(tmp_path / "driver_test")
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Werror", os.path.join(ROOT, "tests", "cpp", "driver_test.cpp"),
                    "-I", INC, "-I", os.path.join(CUDA, "include"), "-L", lib, "-ldgt",
                    "-L", os.path.join(CUDA, "lib64"), "-lcudart", f"-Wl,-rpath,{lib}", "-o", exe], check=True)
    assert os.path.getsize(exe) > 0
