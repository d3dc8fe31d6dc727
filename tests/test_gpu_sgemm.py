"""FP32 GEMM modes through the C ABI against the FP64 oracle of the same FP32 inputs:
3xBF16 split and FP32 SIMT at FP32 accuracy (relative Frobenius <= 1e-5), 1xBF16 at BF16
accuracy (<= 2e-2, and clearly worse than 3xBF16)."""
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


def run(h, mode, ta, tb, m, n, k, alpha=1.0, beta=0.0, seed=0):
    import torch

    ra, ca = (k, m) if ta == "T" else (m, k)
    rb, cb = (n, k) if tb == "T" else (k, n)
    A, B, C = O.normal32((ra, ca), seed + 1), O.normal32((rb, cb), seed + 2), O.normal32((m, n), seed + 3)
    dA, dB, dC = dev(A), dev(B), dev(C)
    h.sgemm(ta, tb, m, n, k, alpha, ptr(dA), ra, ptr(dB), rb, beta, ptr(dC), m, mode=mode)
    torch.cuda.synchronize()
    h.check_device()
    want = O.dgemm(A.astype(np.float64), B.astype(np.float64), alpha, beta, C.astype(np.float64), ta, tb)
    return O.rel_errors(host(dC, (m, n)).astype(np.float64), want)


@pytest.mark.parametrize("ta,tb", [("N", "N"), ("T", "N"), ("N", "T")])
@pytest.mark.parametrize("shape", [(256, 256, 256), (300, 520, 1000), (1, 1, 1), (129, 257, 63)])
def test_sgemm_modes(h, ta, tb, shape):
    m, n, k = shape
    fro3 = run(h, dgt.FP32_BF16X3, ta, tb, m, n, k, 1.5, -0.5)[1]
    fros = run(h, dgt.FP32_SIMT, ta, tb, m, n, k, 1.5, -0.5)[1]
    fro1 = run(h, dgt.FP32_BF16X1, ta, tb, m, n, k, 1.5, -0.5)[1]
    assert fro3 <= 1e-5 and fros <= 1e-5, (fro3, fros)
    assert fro1 <= 2e-2, fro1
    if k >= 63:
        assert fro1 > 10 * fro3, (fro1, fro3)


def test_sgemm_tall_skinny(h):
    """M = N = 4096, K = 512: the tall-skinny shape class of the FP32 configuration."""
    fro3 = run(h, dgt.FP32_BF16X3, "N", "N", 4096, 4096, 512)[1]
    assert fro3 <= 1e-5
