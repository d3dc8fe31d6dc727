"""Ozaki-scheme FP64 emulation on INT8 tcgen05 tensor cores, through the C ABI, against
the host FP64 GEMM oracle.  Tolerances (relative Frobenius vs the oracle): <= 1e-13 at
7-8 slices for U[-1,1) inputs; error must shrink as slices are added."""
import numpy as np
import pytest

import dgt
import oracle as O
from devutil import dev, host, ptr

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def h():
    with dgt.Handle() as handle:
        yield handle


def run(h, ta, tb, m, n, k, alpha, beta, S, A=None, B=None, C=None, mode=dgt.FP64_OZAKI_INT8):
    import torch

    ra, ca = (k, m) if ta == "T" else (m, k)
    rb, cb = (n, k) if tb == "T" else (k, n)
    A = O.uniform((ra, ca), 1) if A is None else A
    B = O.uniform((rb, cb), 2) if B is None else B
    C = O.uniform((m, n), 3) if C is None else C
    dA, dB, dC = dev(A), dev(B), dev(C)
    h.dgemm(ta, tb, m, n, k, alpha, ptr(dA), ra, ptr(dB), rb, beta, ptr(dC), m, mode=mode, slices=S)
    torch.cuda.synchronize()
    h.check_device()
    return host(dC, (m, n)), O.dgemm(A, B, alpha, beta, C, ta, tb)


@pytest.mark.parametrize("ta,tb", [("N", "N"), ("N", "T"), ("T", "N"), ("T", "T")])
@pytest.mark.parametrize("shape", [(256, 256, 128), (300, 200, 100), (1, 1, 1), (129, 513, 1000)])
def test_ozaki_int8_shapes(h, ta, tb, shape):
    m, n, k = shape
    got, want = run(h, ta, tb, m, n, k, 1.5, -0.5, 7)
    _, fro = O.rel_errors(got, want)
    assert fro <= 1e-13, fro


def test_ozaki_error_decreases_with_slices(h):
    errs = []
    for S in (3, 4, 5, 6, 7, 8):
        got, want = run(h, "N", "N", 384, 320, 512, 1.0, 0.0, S)
        errs.append(O.rel_errors(got, want)[1])
    for a, b in zip(errs, errs[1:]):
        assert b < a or b < 1e-15, errs
    assert errs[0] > 1e-7 and errs[-1] < 1e-14, errs


def test_ozaki_wide_dynamic_range_reaches_native_error(h):
    """phi = 4 inputs (entries spread over ~e^+-12): the truncated-digit scheme needs more
    slices than for uniform data.  The Frobenius error keeps falling with S and reaches the
    native DMMA kernel's (both against host OpenBLAS) by 11 slices."""
    import torch

    m = n = k = 512
    A, B = O.ozaki_matrix((m, k), 11, 4.0), O.ozaki_matrix((k, n), 12, 4.0)
    C = np.zeros((m, n), order="F")
    dA, dB, dC = dev(A), dev(B), dev(C)
    h.dgemm("N", "N", m, n, k, 1.0, ptr(dA), m, ptr(dB), k, 0.0, ptr(dC), m, mode=dgt.FP64_NATIVE)
    torch.cuda.synchronize()
    want = A @ B
    nat = O.rel_errors(host(dC, (m, n)), want)[1]
    errs = {}
    for S in (6, 8, 9, 10, 11):
        got, _ = run(h, "N", "N", m, n, k, 1.0, 0.0, S, A, B, C)
        errs[S] = O.rel_errors(got, want)[1]
    assert errs[6] > errs[8] > errs[9], errs
    assert min(errs[10], errs[11]) <= max(2 * nat, 1e-15), (errs, nat)


def test_ozaki_nonfinite_rows_give_nan(h):
    m, n, k = 64, 64, 64
    A = O.uniform((m, k), 1)
    A[5, 7] = np.inf
    got, _ = run(h, "N", "N", m, n, k, 1.0, 0.0, 6, A=A)
    assert np.isnan(got[5, :]).all()
    assert np.isfinite(np.delete(got, 5, axis=0)).all()


def test_ozaki_zero_and_tiny_rows(h):
    m, n, k = 128, 256, 64
    A = O.uniform((m, k), 1)
    A[3, :] = 0.0
    A[4, :] *= 1e-300
    B = O.uniform((k, n), 2)
    got, want = run(h, "N", "N", m, n, k, 1.0, 0.0, 7, A=A, B=B, C=np.zeros((m, n), order="F"))
    assert np.array_equal(got[3, :], np.zeros(n))
    assert O.rel_errors(got[4, :], want[4, :])[1] <= 1e-13
    assert O.rel_errors(got, want)[1] <= 1e-13


def test_ozaki_large_4096(h):
    import torch

    n = 4096
    A, B = O.uniform((n, n), 7), O.uniform((n, n), 8)
    dA, dB = dev(A), dev(B)
    dC = torch.zeros((n, n), dtype=torch.float64, device="cuda")
    h.dgemm("N", "N", n, n, n, 1.0, ptr(dA), n, ptr(dB), n, 0.0, ptr(dC), n, mode=dgt.FP64_OZAKI_INT8, slices=7)
    torch.cuda.synchronize()
    h.check_device()
    got = host(dC, (n, n))
    rows = np.random.default_rng(0).choice(n, 64, replace=False)
    assert O.rel_errors(got[rows, :], A[rows, :] @ B)[1] <= 1e-13


@pytest.mark.parametrize("variant", [0, 1, 2, 3, 4, 5, 6, 7])
def test_ozaki_kernel_variants(variant):
    """Every tuning variant of the INT8 kernel (epilogue warps x stage depth, and the CTA-pair
    kernel with 256 x 256 tiles) gives the same digits-exact products: identical to variant 0,
    and within 1e-13 of the oracle."""
    import torch

    m, n, k = 300, 520, 1000
    A, B, C = O.uniform((m, k), 41), O.uniform((k, n), 42), O.uniform((m, n), 43)
    outs = []
    for v in (0, variant):
        with dgt.Handle() as hh:
            hh.set_tuning(dgt.TUNE_OZAKI_VARIANT, v)
            dA, dB, dC = dev(A), dev(B), dev(C)
            hh.dgemm("N", "N", m, n, k, 1.25, ptr(dA), m, ptr(dB), k, 0.5, ptr(dC), m, mode=dgt.FP64_OZAKI_INT8,
                     slices=7)
            torch.cuda.synchronize()
            hh.check_device()
            outs.append(host(dC, (m, n)))
    assert np.array_equal(outs[0], outs[1])
    assert O.rel_errors(outs[1], O.dgemm(A, B, 1.25, 0.5, C))[1] <= 1e-13


@pytest.mark.parametrize("shape", [(256, 256, 128), (300, 200, 2500), (1, 1, 1)])
def test_ozaki_bf16_slices(h, shape):
    """BF16 digit planes with exact FP32 accumulation (flushed every 1024 of K) give the
    same accuracy as the INT8 planes."""
    m, n, k = shape
    got16, want = run(h, "N", "N", m, n, k, 1.5, -0.5, 7, mode=dgt.FP64_OZAKI_BF16)
    got8, _ = run(h, "N", "N", m, n, k, 1.5, -0.5, 7)
    assert O.rel_errors(got16, want)[1] <= 1e-13
    assert O.rel_errors(got16, got8)[1] <= 1e-14
