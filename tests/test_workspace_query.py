"""dgt_dgemm_workspace_size (no handle, no device call): the CRT workspace equals the
restated layout (planes of op(A) and op(B), amax words and norm bounds, exponents, residue
planes of C, each rounded up to 1 KB; the CTA-pair variant pads M to 256; K is one chunk of at
most 65536), the slice workspace covers its digit planes, and bad counts are rejected."""
import ctypes
import sys

import pytest

sys.path.insert(0, "distributed-gemm-thesis_b200")
import dgt  # noqa: E402


def _up(x):
    return (x + 1023) // 1024 * 1024


def _cd(a, b):
    return -(-a // b) * b


def _crt_bytes(nmod, m, n, k):
    kc = min(max(k, 1), 65536)
    best = 0
    for unit in (128, 256):
        m_pad, n_pad, k_pad = _cd(m, unit), _cd(n, 256), _cd(kc, 128)
        pa, pb = _up(nmod * m_pad * k_pad), _up(nmod * n_pad * k_pad)
        xa, xb, ea, eb = _up(m * 8), _up(n * 8), _up(m * 4), _up(n * 4)
        rs = _up(nmod * m_pad * n_pad)
        sc = 1024  # the residue GEMM's unit counter
        best = max(best, pa + pb + 2 * (xa + xb) + ea + eb + rs + sc)
    return best


@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (1000, 900, 777), (16384, 16384, 16384), (300, 5000, 70000)])
@pytest.mark.parametrize("nmod", [8, 14, 16, 20])
def test_crt_workspace_matches_layout(m, n, k, nmod):
    assert dgt.dgemm_workspace_size(m, n, k, dgt.FP64_OZAKI2_INT8, nmod) == _crt_bytes(nmod, m, n, k)


def test_slices_and_auto_and_native():
    m, n, k = 2000, 3000, 4000
    planes = lambda S, e: S * (_cd(m, 128) * _cd(k, 128) + _cd(n, 256) * _cd(k, 128)) * e
    s7 = dgt.dgemm_workspace_size(m, n, k, dgt.FP64_OZAKI_INT8, 7)
    s8 = dgt.dgemm_workspace_size(m, n, k, dgt.FP64_OZAKI_INT8, 8)
    assert planes(7, 1) <= s7 < s8
    assert dgt.dgemm_workspace_size(m, n, k, dgt.FP64_OZAKI_BF16, 7) >= planes(7, 2)
    # AUTO: the larger of the INT8-slice and CRT workspaces for the count (8 is also a modulus
    # count; 7 is not, so the CRT candidate takes 16 moduli, as the autotuner does)
    assert dgt.dgemm_workspace_size(m, n, k, dgt.FP64_AUTO, 8) == max(s8, _crt_bytes(8, m, n, k))
    assert dgt.dgemm_workspace_size(m, n, k, dgt.FP64_AUTO, 7) == max(s7, _crt_bytes(16, m, n, k))
    assert dgt.dgemm_workspace_size(m, n, k, dgt.FP64_NATIVE, 0) == 0
    assert dgt.dgemm_workspace_size(m, 0, k, dgt.FP64_OZAKI2_INT8, 16) == 0


def test_rejections():
    lib = dgt.load()
    out = ctypes.c_size_t()
    assert lib.dgt_dgemm_workspace_size(10, 10, 10, dgt.FP64_OZAKI2_INT8, 7, ctypes.byref(out)) == 1  # < 8 moduli
    assert lib.dgt_dgemm_workspace_size(10, 10, 10, dgt.FP64_OZAKI_INT8, 1, ctypes.byref(out)) == 1  # < 2 slices
    assert lib.dgt_dgemm_workspace_size(-1, 10, 10, dgt.FP64_OZAKI_INT8, 7, ctypes.byref(out)) == 1
    assert lib.dgt_dgemm_workspace_size(10, 10, 10, dgt.FP64_OZAKI_INT8, 7, None) == 1
