"""dgt_dgemm_ozaki_static: the FP64-accurate (INT8 Ozaki) GEMM for callers that cannot
allocate device memory when they multiply (under a foreign allocator that owns the device
memory, in allocation-free real-time loops).  Its scratch is a fixed 64 MiB device array
inside the library.  Checked through the C ABI against the handle-based entry point
(dgt_dgemm_ex, same slice count) on calls in a row, so each later call runs on scratch an
earlier, larger one left behind; the tolerance is the one the Ozaki tests use (relative
Frobenius <= 1e-13).  Both operand layouts are covered (op(A) K-contiguous with 'T'), with
odd sizes.  After the calls, dgt_ozaki_static_check reads the sticky device error word:
clean.  This file is collected last of the GPU suite."""
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


def _check_entry():
    lib = dgt.load()
    fn = lib.dgt_ozaki_static_check
    fn.restype = ctypes.c_int32
    fn.argtypes = [ctypes.c_void_p]
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


def test_static_scratch_matches_handle_entry_in_a_row():
    import torch

    fn, check = _entry(), _check_entry()
    with dgt.Handle() as h:
        _case(fn, h, "N", "T", 300, 200, 100, 1.5, -0.5, 7, 11)
        _case(fn, h, "N", "N", 256, 513, 640, 1.0, 0.0, 8, 21)
        _case(fn, h, "T", "N", 129, 77, 301, -0.75, 0.25, 7, 31)  # smaller, on the larger call's leftovers
        _case(fn, h, "T", "T", 65, 143, 97, 1.0, 2.0, 8, 41)
    assert check(torch.cuda.current_stream().cuda_stream) == dgt.SUCCESS


def test_static_k_zero_scales_c():
    import torch

    fn = _entry()
    m, n = 37, 21
    C = O.uniform((m, n), 51)
    dC = dev(C)
    a, b = ctypes.c_double(1.0), ctypes.c_double(-0.5)
    x = torch.zeros(1, dtype=torch.float64, device="cuda")
    st = fn(torch.cuda.current_stream().cuda_stream, b"N", b"N", m, n, 0, ctypes.byref(a), ptr(x), m, ptr(x), 1,
            ctypes.byref(b), ptr(dC), m, 7)
    assert st == dgt.SUCCESS
    torch.cuda.synchronize()
    assert np.array_equal(host(dC, (m, n)), -0.5 * C)


def test_static_scratch_rejects_oversize():
    import torch

    fn = _entry()
    a, b = ctypes.c_double(1.0), ctypes.c_double(0.0)
    x = torch.zeros(1, dtype=torch.float64, device="cuda")
    # 8192^3 at 7 slices needs ~940 MiB of digit planes: more than the 64 MiB array
    st = fn(0, b"N", b"N", 8192, 8192, 8192, ctypes.byref(a), ptr(x), 8192, ptr(x), 8192, ctypes.byref(b), ptr(x),
            8192, 7)
    assert st == dgt.INVALID_VALUE
