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
    assert list(full["M"]) == [64, 64, 96, 64] and list(full["StackSize"]) == [1, 1, 2, 1]
    assert list(pre["M"]) == [96] and list(pre["dRow"]) == [4]
    for df in (full, pre):
        assert (df["Algo"] == "2.5D CANNON dgt").all()
        assert (df["DataLocation"] == "devices").all() and (df["TotalGPUs"] == 1).all()
        assert (df["ExecutionTime"] > 0).all() and (df["GFlops"] > 0).all()
        assert (df["GemmCallTime"] == df["ExecutionTime"]).all() and (df["CommunicationTime"] == 0).all()


class HostOps:
    """Rank-local operations on CPU tensors: the test double of dgt.dist.DgtOps for the
    multi-process schedules run as gloo ranks.  Like dgt_dgemm, C is not read when beta
    is 0."""

    def empty(self, shape, like):
        import torch

        return torch.empty(shape, dtype=torch.float64)

    def pack_rows(self, src, r0, rows, dst):
        dst.copy_(src[:, r0:r0 + rows])

    def copy(self, src, dst):
        dst.copy_(src)

    def gemm(self, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc):
        c = C.numpy()[:n, :m]  # column-major m x n view of C's storage
        prod = A.numpy()[:k, :m].T @ B.numpy()[:n, :k].T if k > 0 else np.zeros((m, n))
        c[...] = (alpha * prod).T if beta == 0.0 else (alpha * prod + beta * c.T).T
