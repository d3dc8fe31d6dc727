"""dgt_dgemm_host: A, B and C in host memory, copies pipelined with the computation in column
panels (and, in the CRT mode with a tall op(A), in a 2D order of row and column panels).  In the CRT mode op(A) is split once and every panel's result equals the
whole-matrix device call bit for bit (row scaling depends on op(A)'s rows alone, column
scaling on op(B)'s columns alone); other modes run the device GEMM per panel.  Page-locked and
pageable host buffers give the same results (pageable ones only serialize the copies)."""
import numpy as np
import pytest

import dgt
import oracle as O
from devutil import dev, host, ptr

pytestmark = pytest.mark.gpu
FRO_TOL = 1e-13


def _pinned(a):
    """A page-locked host copy of column-major `a` (torch owns the memory) and its address."""
    import torch

    a = np.asfortranarray(a)
    t = torch.from_numpy(np.ascontiguousarray(a.T)).pin_memory()
    return t, t.data_ptr()


def _case(m, n, k, ta, tb, seed):
    A = O.uniform((k, m) if ta == "T" else (m, k), seed)
    B = O.uniform((n, k) if tb == "T" else (k, n), seed + 1)
    C = O.uniform((m, n), seed + 2)
    return A, B, C


def _device_result(h, A, B, C, ta, tb, m, n, k, alpha, beta, mode, S):
    import torch

    dA, dB, dC = dev(A), dev(B), dev(C)
    h.dgemm(ta, tb, m, n, k, alpha, ptr(dA), A.shape[0], ptr(dB), B.shape[0], beta, ptr(dC), m, mode=mode, slices=S)
    torch.cuda.synchronize()
    h.check_device()
    return host(dC, (m, n))


def _host_result(h, A, B, C, ta, tb, m, n, k, alpha, beta, mode, S, panel_cols, pinned=True):
    import torch

    if pinned:
        tA, pA = _pinned(A)
        tB, pB = _pinned(B)
        tC, pC = _pinned(C)
    else:  # pageable numpy buffers
        tA, tB, tC = np.asfortranarray(A), np.asfortranarray(B), np.asfortranarray(C.copy())
        pA, pB, pC = tA.ctypes.data, tB.ctypes.data, tC.ctypes.data
    h.dgemm_host(ta, tb, m, n, k, alpha, pA, A.shape[0], pB, B.shape[0], beta, pC, m, mode=mode, slices=S,
                 panel_cols=panel_cols)
    torch.cuda.synchronize()
    h.check_device()
    if pinned:
        return np.asfortranarray(tC.numpy().T)
    return tC


@pytest.mark.parametrize("m,n,k,ta,tb,beta,panel", [
    (1000, 2300, 777, "N", "N", -0.5, 512),   # ragged last panel, C read
    (333, 1100, 2049, "T", "N", 0.0, 256),
    (700, 900, 300, "N", "T", 1.25, 0),       # automatic panel width (one panel)
    (517, 1300, 1000, "T", "T", 0.0, 384),
])
def test_crt_host_equals_device_bitwise(m, n, k, ta, tb, beta, panel):
    A, B, C = _case(m, n, k, ta, tb, 7 * m + n)
    with dgt.Handle() as h:
        want = _device_result(h, A, B, C, ta, tb, m, n, k, 1.5, beta, dgt.FP64_OZAKI2_INT8, 16)
        got = _host_result(h, A, B, C, ta, tb, m, n, k, 1.5, beta, dgt.FP64_OZAKI2_INT8, 16, panel)
    assert np.array_equal(got, want)
    ref = O.dgemm(A, B, 1.5, beta, C, ta, tb)
    assert O.rel_errors(got, ref)[1] <= FRO_TOL


@pytest.mark.parametrize("m,n,k,ta,tb,beta,panel", [
    (2600, 2300, 777, "N", "N", -0.5, 512),   # 3 row panels x 5 column panels, both ragged, C read
    (2100, 1000, 300, "T", "T", 0.0, 0),      # automatic column width
    (3000, 700, 2049, "N", "T", 1.25, 256),
    (2049, 1300, 1000, "T", "N", 0.0, 384),   # a one-row last panel
])
def test_crt_host_2d_block_order_equals_device_bitwise(m, n, k, ta, tb, beta, panel):
    """A tall op(A) runs in 2D block order: row panels of op(A) and column panels of op(B)
    arrive alternately, each is split on arrival, and every completed C block is computed and
    sent back.  Bit for bit the whole-matrix device call."""
    A, B, C = _case(m, n, k, ta, tb, 3 * m + n)
    with dgt.Handle() as h:
        want = _device_result(h, A, B, C, ta, tb, m, n, k, 1.5, beta, dgt.FP64_OZAKI2_INT8, 15)
        got = _host_result(h, A, B, C, ta, tb, m, n, k, 1.5, beta, dgt.FP64_OZAKI2_INT8, 15, panel)
    assert np.array_equal(got, want)
    assert O.rel_errors(got, O.dgemm(A, B, 1.5, beta, C, ta, tb))[1] <= FRO_TOL


def test_host_pageable_equals_pinned():
    m, n, k = 640, 1500, 900
    A, B, C = _case(m, n, k, "N", "N", 41)
    with dgt.Handle() as h:
        pinned = _host_result(h, A, B, C, "N", "N", m, n, k, 1.0, 0.5, dgt.FP64_OZAKI2_INT8, 16, 512)
        pageable = _host_result(h, A, B, C, "N", "N", m, n, k, 1.0, 0.5, dgt.FP64_OZAKI2_INT8, 16, 512, pinned=False)
    assert np.array_equal(pinned, pageable)


@pytest.mark.parametrize("mode,S", [(dgt.FP64_NATIVE, 7), (dgt.FP64_OZAKI_INT8, 8)])
def test_other_modes_per_panel(mode, S):
    """Native DMMA and the slice scheme run the device GEMM on each panel: within 1e-13 of the
    host FP64 GEMM, and equal to the whole-matrix device call column block by column block."""
    m, n, k = 800, 1700, 640
    A, B, C = _case(m, n, k, "N", "T", 77)
    with dgt.Handle() as h:
        got = _host_result(h, A, B, C, "N", "T", m, n, k, -1.0, 0.25, mode, S, 512)
        want = _device_result(h, A, B, C, "N", "T", m, n, k, -1.0, 0.25, mode, S)
    ref = O.dgemm(A, B, -1.0, 0.25, C, "N", "T")
    assert O.rel_errors(got, ref)[1] <= FRO_TOL
    assert O.rel_errors(got, want)[1] <= FRO_TOL


def test_crt_long_k_per_panel():
    """K beyond one exact residue product: each panel runs the K-chunked device path."""
    m, n, k = 64, 600, 70000
    A, B, C = _case(m, n, k, "N", "N", 5)
    with dgt.Handle() as h:
        got = _host_result(h, A, B, C, "N", "N", m, n, k, 1.0, 0.0, dgt.FP64_OZAKI2_INT8, 16, 256)
        want = _device_result(h, A, B, C, "N", "N", m, n, k, 1.0, 0.0, dgt.FP64_OZAKI2_INT8, 16)
    assert np.array_equal(got, want)


def test_host_edge_cases():
    """k = 0 gives C = beta C; m = 0 touches nothing; a null alpha is rejected."""
    import ctypes

    m, n = 90, 130
    C = O.uniform((m, n), 9)
    with dgt.Handle() as h:
        got = _host_result(h, np.zeros((m, 1)), np.zeros((1, n)), C, "N", "N", m, n, 0, 1.0, 0.5,
                           dgt.FP64_OZAKI2_INT8, 16, 64)
        assert np.array_equal(got, 0.5 * C)
        tC, pC = _pinned(C)
        h.dgemm_host("N", "N", 0, n, 5, 1.0, pC, 1, pC, 5, 0.0, pC, 1, mode=dgt.FP64_OZAKI2_INT8, slices=16)
        assert np.array_equal(np.asfortranarray(tC.numpy().T), C)
        b = ctypes.c_double(0.0)
        st = h.lib.dgt_dgemm_host(h.h, b"N", b"N", m, n, 4, None, pC, m, pC, 4, ctypes.byref(b), pC, m,
                                  dgt.FP64_OZAKI2_INT8, 16, 0)
        assert st == 1  # DGT_ERROR_INVALID_VALUE
