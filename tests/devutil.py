"""Helpers shared by the tests: column-major numpy <-> device memory owned by torch (torch
only owns the memory; every computation goes through libdgt), the CSV-log checks of the
C++ drivers, and the host doubles of the multi-process tests (rank-local operations,
process-shared memory standing in for CUDA IPC, block-cyclic scatter / gather, free ports)."""
import ctypes
import socket

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

def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def scatter_block_cyclic(G, mb, nb, p, q):
    """Block-cyclic locals of every rank of a p x q grid (rank r = i q + j), empty ranks
    included (the oracle's scatter refuses grids that leave a rank empty)."""
    M, N = G.shape
    out = []
    for r in range(p * q):
        i, j = r // q, r % q
        rows = [x for b in range(i, -(-M // mb), p) for x in range(b * mb, min(M, (b + 1) * mb))]
        cols = [x for b in range(j, -(-N // nb), q) for x in range(b * nb, min(N, (b + 1) * nb))]
        out.append(np.asfortranarray(G[np.ix_(rows, cols)]))
    return out


def gather_block_cyclic(locs, M, N, mb, nb, p, q):
    G = np.full((M, N), np.nan)
    for r, loc in enumerate(locs):
        i, j = r // q, r % q
        rows = [x for b in range(i, -(-M // mb), p) for x in range(b * mb, min(M, (b + 1) * mb))]
        cols = [x for b in range(j, -(-N // nb), q) for x in range(b * nb, min(N, (b + 1) * nb))]
        G[np.ix_(rows, cols)] = loc
    return G


def local_tensor(x):
    import torch

    rows, cols = x.shape
    t = torch.zeros((max(cols, 1), max(rows, 1)), dtype=torch.float64)
    if rows and cols:
        t.copy_(torch.from_numpy(np.ascontiguousarray(np.asfortranarray(x).T)))
    return t


class ShmIpc:
    """Host shared memory with DeviceIpc's interface (alloc / open / close / free / tensor)."""

    def __init__(self):
        self.segments = {}

    def _addr(self, shm):
        return np.frombuffer(shm.buf, dtype=np.uint8).ctypes.data

    def alloc(self, nbytes):
        from multiprocessing import shared_memory

        shm = shared_memory.SharedMemory(create=True, size=max(int(nbytes), 8))
        addr = self._addr(shm)
        self.segments[addr] = shm
        return addr, shm.name.encode().ljust(64, b"\0")

    def open(self, handle):
        from multiprocessing import shared_memory

        shm = shared_memory.SharedMemory(name=handle.rstrip(b"\0").decode())
        addr = self._addr(shm)
        self.segments[addr] = shm
        return addr

    def close(self, ptr):
        pass  # mappings go with the process

    def free(self, ptr):
        self.segments[ptr].unlink()

    def tensor(self, ptr, shape):
        import torch

        n = int(np.prod(shape))
        return torch.from_numpy(np.frombuffer((ctypes.c_double * n).from_address(ptr), dtype=np.float64).reshape(shape))

    def synchronize(self):
        pass


class CannonHandle:
    """dgt.Handle.cannon25d_rank and reduce_tiles executed on host addresses."""

    @staticmethod
    def _mat(addr, rows, cols, ld):
        n = ld * (cols - 1) + rows
        buf = np.frombuffer((ctypes.c_double * n).from_address(addr), dtype=np.float64)
        return np.lib.stride_tricks.as_strided(buf, shape=(rows, cols), strides=(8, 8 * ld))

    def cannon25d_rank(self, M, p, c, rank, alpha, A_tiles, B_tiles, beta, C_tile, ta="N", tb="N", mode=None,
                       slices=7):
        import dgt

        lm = M // p
        k, i, j = rank // (p * p), (rank // p) % p, rank % p
        order, _ = dgt.cannon_schedule(p, c, i, j, k)
        acc = np.zeros((lm, lm))
        for t in order:
            acc += self._mat(A_tiles[i * p + t], lm, lm, lm) @ self._mat(B_tiles[t * p + j], lm, lm, lm)
        C = self._mat(C_tile, lm, lm, lm)
        C[...] = alpha * acc + (beta * C if k == 0 and beta != 0.0 else 0.0)

    def reduce_tiles(self, C, parts, elems):
        c = self._mat(C, elems, 1, elems)
        for part in parts:
            c += self._mat(part, elems, 1, elems)


class ScheduleHandle:
    """dgt.Handle.summa_rank executed on host addresses: the segments dgt_summa_schedule
    returns, each a rank-local GEMM reading the owners' memory."""

    @staticmethod
    def _mat(addr, rows, cols, ld):
        n = ld * (cols - 1) + rows if rows and cols else 1
        buf = np.frombuffer((ctypes.c_double * n).from_address(addr), dtype=np.float64)
        return np.lib.stride_tricks.as_strided(buf, shape=(rows, cols), strides=(8, 8 * ld))

    def summa_rank(self, rank, p, q, mb, nb, kb, M, N, K, alpha, A_ptrs, lldA, B_ptrs, lldB, beta, C, ldc,
                   mode=None, slices=7):
        import dgt

        m, n = dgt.numroc(M, mb, rank // q, 0, p), dgt.numroc(N, nb, rank % q, 0, q)
        if m == 0 or n == 0:
            return
        c = self._mat(C, m, n, ldc)
        first = True
        for a, b, lda, ldb, k in dgt.summa_schedule(rank, p, q, mb, nb, kb, M, N, K, A_ptrs, lldA, B_ptrs, lldB):
            prod = self._mat(a, m, k, lda) @ self._mat(b, k, n, ldb) if k else 0.0
            c[...] = alpha * prod + (beta if first else 1.0) * c
            first = False
