"""dgt_dgemm_ozaki_static: the FP64-accurate (INT8 Ozaki) GEMM for callers that cannot
allocate device memory when they multiply (under a foreign allocator that owns the device
memory, in allocation-free real-time loops).  Its scratch is
a fixed 64 MiB device array inside the library.  Checked through the C ABI against the
handle-based entry point (dgt_dgemm_ex, same slice count) on two calls in a row, so the
second call runs on scratch the first one left behind; the tolerance is the one the Ozaki
tests use (relative Frobenius <= 1e-13).  Collected after the rest of the validated GPU
suite, before the tests of the newest entries."""
import ctypes

import numpy as np
import pytest

import dgt
import oracle as O
from devutil import dev, host, ptr

pytestmark = pytest.mark.gpu
TOL = 1e-13


def _entry():
    lib = dgt.load()
    fn = lib.dgt_dgemm_ozaki_static
    fn.restype = ctypes.c_int32
    fn.argtypes = [ctypes.c_void_p, ctypes.c_char, ctypes.c_char, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64,
                   ctypes.POINTER(ctypes.c_double), ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64,
                   ctypes.POINTER(ctypes.c_double), ctypes.c_void_p, ctypes.c_int64, ctypes.c_int]
    return fn


def _case(fn, h, ta, tb, m, n, k, alpha, beta, S, seed):
    import torch

    ra, ca = (k, m) if ta == "T" else (m, k)
    rb, cb = (n, k) if tb == "T" else (k, n)
    A, B, C = O.uniform((ra, ca), seed), O.uniform((rb, cb), seed + 1), O.uniform((m, n), seed + 2)
    dA, dB = dev(A), dev(B)
    dC_static, dC_ref = dev(C), dev(C)
    stream = torch.cuda.current_stream().cuda_stream
    a, b = ctypes.c_double(alpha), ctypes.c_double(beta)
    st = fn(stream, ta.encode(), tb.encode(), m, n, k, ctypes.byref(a), ptr(dA), ra, ptr(dB), rb, ctypes.byref(b),
            ptr(dC_static), m, S)
    assert st == dgt.SUCCESS, st
    h.set_stream(stream)
    h.dgemm(ta, tb, m, n, k, alpha, ptr(dA), ra, ptr(dB), rb, beta, ptr(dC_ref), m, mode=dgt.FP64_OZAKI_INT8, slices=S)
    torch.cuda.synchronize()
    got, ref = host(dC_static, (m, n)), host(dC_ref, (m, n))
    assert O.rel_errors(got, ref)[1] <= TOL
    assert O.rel_errors(got, O.dgemm(A, B, alpha, beta, C, ta, tb))[1] <= TOL


def test_static_scratch_matches_handle_entry_twice():
    fn = _entry()
    with dgt.Handle() as h:
        _case(fn, h, "N", "T", 300, 200, 100, 1.5, -0.5, 7, 11)
        _case(fn, h, "N", "N", 256, 513, 640, 1.0, 0.0, 8, 21)


def test_static_scratch_rejects_oversize():
    import torch

    fn = _entry()
    a, b = ctypes.c_double(1.0), ctypes.c_double(0.0)
    x = torch.zeros(1, dtype=torch.float64, device="cuda")
    # 8192^3 at 7 slices needs ~940 MiB of digit planes: more than the 64 MiB array
    st = fn(0, b"N", b"N", 8192, 8192, 8192, ctypes.byref(a), ptr(x), 8192, ptr(x), 8192, ctypes.byref(b), ptr(x),
            8192, 7)
    assert st == dgt.INVALID_VALUE
