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
