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


def _csv_format(tmp_path):
    exe = str(tmp_path / "csv_format")
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Werror", os.path.join(ROOT, "tests", "cpp", "csv_format.cpp"),
                    "-I", INC, "-o", exe], check=True)
    return lambda *args, stdin=None: subprocess.run([exe, *args], input=stdin, capture_output=True, text=True,
                                                    timeout=60, check=True).stdout


def test_logger_matches_reference_logging(tmp_path):
    """Against the reference's own fullOffloadSumma25Dgemm with logging on (compiled from its
    sources into oracle/_ref with MACHINE_NAME "oracle"): same file name, header written
    once across two calls, every row it wrote printed identically by dgt::cannonCsvLine from
    the row's own values, and the same file after createLogCsv on a log whose first line is
    another header."""
    import numpy as np

    import oracle as O

    if not O.ref_available():
        pytest.skip("oracle/_ref not built (reference sources absent)")
    fmt = _csv_format(tmp_path)
    R = O.ref()
    R.use_naive()
    name = fmt("name", "full", "oracle", "cuBLAS").strip()
    assert name == "DGEMM_execution_logs-FullOffload_GEMM-oracle-2.5DCANNON-cuBLAS.csv"

    d1 = tmp_path / "ref1"
    d1.mkdir()
    A, B, C = (O.uniform((16, 16), s) for s in (1, 2, 3))
    out = R.cannon_fulloffload_logged(d1, A, B, C, 2, 1, 1.0, 0.0, 2)
    R.cannon_fulloffload_logged(d1, A, B, C, 4, 2, 1.0, 0.0, 1)
    assert sorted(os.listdir(d1)) == [name]
    text = (d1 / name).read_text()
    lines = text.splitlines(keepends=True)
    assert lines[0] == fmt("header")
    assert text.count("Algo,") == 1 and len(lines) == 4
    assert fmt("rows", stdin="".join(lines[1:])) == "".join(lines[1:])
    # the reference's runs after the first start from tiles its previous multiply left
    # rotated, so only a single run gives A B (the drivers here multiply the original tiles
    # on every run)
    single = R.cannon_fulloffload_logged(d1, A, B, C, 2, 1, 1.0, 0.0, 1)
    assert np.abs(single - A @ B).max() < 1e-12 and np.abs(out - A @ B).max() > 1e-3

    foreign = "Algo,M,N,K\nx,1,2,3\n"
    d2 = tmp_path / "ref2"
    d2.mkdir()
    (d2 / name).write_text(foreign)
    R.cannon_fulloffload_logged(d2, A, B, C, 2, 1, 1.0, 0.0, 1)
    ours = tmp_path / "ours.csv"
    ours.write_text(foreign)
    fmt("open", str(ours))
    ref_text, our_text = (d2 / name).read_text(), ours.read_text()
    assert ref_text.startswith(our_text) and our_text == foreign + fmt("header")
    assert ref_text[len(our_text):].count("\n") == 1
