"""Device-buffer helpers for the GPU tests: column-major numpy <-> device memory owned
by torch (torch only owns the memory; every computation goes through libdgt)."""
import numpy as np


def dev(a):
    import torch

    a = np.asfortranarray(a)
    return torch.from_numpy(np.ascontiguousarray(a.T)).cuda()


def host(t, shape):
    arr = t.cpu().numpy()
    return np.asfortranarray(arr.T.reshape(shape, order="F")) if arr.ndim == 2 else arr.reshape(shape, order="F")


def zeros(rows, cols, dtype=None):
    import torch

    return torch.zeros((max(cols, 1), max(rows, 1)), dtype=dtype or torch.float64, device="cuda")


def ptr(t):
    return t.data_ptr()


def check_cannon_driver_logs(logs):
    """CSV rows that tests/cpp/driver_test.cpp makes the 2.5D Cannon drivers write, read the
    way the thesis notebooks read them (pandas.read_csv, header=0)."""
    import pandas as pd

    full = pd.read_csv(logs / "DGEMM_execution_logs-FullOffload_GEMM-b200test-2.5DCANNON-dgt.csv", header=0)
    pre = pd.read_csv(logs / "DGEMM_execution_logs-PreDistributed_GEMM-b200test-2.5DCANNON-dgt.csv", header=0)
    assert list(full["M"]) == [64, 64, 96] and list(full["StackSize"]) == [1, 1, 2]
    assert list(pre["M"]) == [96] and list(pre["dRow"]) == [4]
    for df in (full, pre):
        assert (df["Algo"] == "2.5D CANNON dgt").all()
        assert (df["DataLocation"] == "devices").all() and (df["TotalGPUs"] == 1).all()
        assert (df["ExecutionTime"] > 0).all() and (df["GFlops"] > 0).all()
        assert (df["GemmCallTime"] == df["ExecutionTime"]).all() and (df["CommunicationTime"] == 0).all()
