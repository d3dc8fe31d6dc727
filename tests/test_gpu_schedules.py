"""In-device step schedules through the C ABI: SUMMA on block-cyclic local buffers,
2.5D Cannon on equal tiles, and the grouped persistent launch -- against the host FP64
GEMM oracle (relative Frobenius <= 1e-13) and, for Cannon, the reference's own result."""
import os

import numpy as np
import pytest

import dgt
import oracle as O
from devutil import dev, host, ptr

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FRO_TOL = 1e-13


@pytest.fixture(scope="module")
def h():
    with dgt.Handle() as handle:
        yield handle


def summa_run(h, M, N, K, b, p, q, alpha, beta, seeds=(1, 2, 3), sample_rows=None):
    """Packs A, B, C block-cyclically (the product's pack), runs dgt_summa, unpacks C."""
    import torch

    A, B, C = O.uniform((M, K), seeds[0]), O.uniform((K, N), seeds[1]), O.uniform((M, N), seeds[2])
    o = O.orc()

    def pack(X, rows, cols):
        shapes = o.pblas_shapes(rows, cols, b, b, p, q)
        locs = [torch.zeros((max(c, 1), max(r, 1)), dtype=torch.float64, device="cuda") for r, c, _ in shapes]
        lld = [max(r, 1) for r, _, _ in shapes]
        dX = dev(X)
        h.pack_block_cyclic(rows, cols, b, b, p, q, ptr(dX), rows, [ptr(l) for l in locs], lld)
        return dX, locs, lld

    _, lA, lldA = pack(A, M, K)
    _, lB, lldB = pack(B, K, N)
    dC, lC, lldC = pack(C, M, N)
    h.summa(p, q, b, b, b, M, N, K, alpha, [ptr(x) for x in lA], lldA, [ptr(x) for x in lB], lldB, beta,
            [ptr(x) for x in lC], lldC)
    h.unpack_block_cyclic(M, N, b, b, p, q, ptr(dC), M, [ptr(x) for x in lC], lldC)
    torch.cuda.synchronize()
    h.check_device()
    got = host(dC, (M, N))
    if sample_rows is None:
        return O.rel_errors(got, O.dgemm(A, B, alpha, beta, C))
    rows = np.sort(np.random.default_rng(7).choice(M, sample_rows, replace=False))
    want = alpha * (A[rows, :] @ B) + beta * C[rows, :]
    return O.rel_errors(got[rows, :], want)


@pytest.mark.parametrize("M,N,K,b,p,q", [(64, 64, 64, 16, 2, 2), (100, 90, 77, 8, 3, 2), (257, 131, 199, 32, 2, 3),
                                         (500, 400, 300, 64, 4, 4)])
def test_summa_small(h, M, N, K, b, p, q):
    _, fro = summa_run(h, M, N, K, b, p, q, 1.5, -0.5)
    assert fro <= FRO_TOL


def test_summa_config1(h):
    """4096^3, 2 x 2 grid, 512 blocks, alpha = 1, beta = 0."""
    _, fro = summa_run(h, 4096, 4096, 4096, 512, 2, 2, 1.0, 0.0, seeds=(20261203, 20261204, 20261205))
    assert fro <= FRO_TOL


def test_summa_config2_ragged(h):
    """M=15000, N=17000, K=9000, 4 x 4 grid, block 256, alpha=1.5, beta=-0.5 (sampled rows)."""
    _, fro = summa_run(h, 15000, 17000, 9000, 256, 4, 4, 1.5, -0.5, sample_rows=96)
    assert fro <= FRO_TOL


def cannon_run(h, M, p, c, alpha, beta, A, B, C):
    import torch

    dA, dB, dC = dev(A), dev(B), dev(C)
    lm = M // p
    tiles = lambda: [torch.zeros((lm, lm), dtype=torch.float64, device="cuda") for _ in range(p * p)]
    tA, tB, tC = tiles(), tiles(), tiles()
    h.pack_cannon2d(M, p, ptr(dA), ptr(dB), ptr(dC), [ptr(x) for x in tA], [ptr(x) for x in tB],
                    [ptr(x) for x in tC])
    h.cannon25d(M, p, c, alpha, [ptr(x) for x in tA], [ptr(x) for x in tB], beta, [ptr(x) for x in tC])
    h.unpack_cannon2d(M, p, ptr(dC), [ptr(x) for x in tC])
    torch.cuda.synchronize()
    h.check_device()
    return host(dC, (M, M))


def test_cannon_against_reference_golden(h):
    g = np.load(os.path.join(GOLD, "cannon.npz"))
    idx = 0
    while f"cannon{idx}_params" in g:
        M, p, c = (int(v) for v in g[f"cannon{idx}_params"])
        A, B, C = g[f"cannon{idx}_A"], g[f"cannon{idx}_B"], g[f"cannon{idx}_C"]
        got = cannon_run(h, M, p, c, 1.5, -0.5, A, B, C)
        want = O.dgemm(A, B, 1.5, -0.5, C)
        assert O.rel_errors(got, want)[1] <= FRO_TOL, (M, p, c)
        ref_fro = O.rel_errors(g[f"cannon{idx}_result"], want)[1]
        if ref_fro < 1e-14:  # where the reference is right, we agree with it
            assert O.rel_errors(got, g[f"cannon{idx}_result"])[1] <= FRO_TOL
        idx += 1


@pytest.mark.parametrize("M,p,c", [(512, 4, 2), (1024, 4, 1), (768, 3, 1), (1200, 6, 2), (2048, 8, 4)])
def test_cannon_shapes(h, M, p, c):
    A, B, C = O.uniform((M, M), 1), O.uniform((M, M), 2), O.uniform((M, M), 3)
    got = cannon_run(h, M, p, c, 1.0, 1.0, A, B, C)
    assert O.rel_errors(got, O.dgemm(A, B, 1.0, 1.0, C))[1] <= FRO_TOL


def test_grouped_ragged_products(h):
    """48 independent products, M, N, K log-uniform in [1, 700], in one launch."""
    import torch

    rng = np.random.default_rng(5)
    descs, keep = [], []
    for i in range(48):
        m, n, k = (int(round(np.exp(rng.uniform(0, np.log(700))))) for _ in range(3))
        A, B, C = O.uniform((m, k), 100 + i), O.uniform((k, n), 200 + i), O.uniform((m, n), 300 + i)
        dA, dB, dC = dev(A), dev(B), dev(C)
        al, be = float(rng.uniform(-2, 2)), float(rng.uniform(-1, 1))
        descs.append(dict(m=m, n=n, k=k, alpha=al, beta=be, A=ptr(dA), lda=m, B=ptr(dB), ldb=k, C=ptr(dC), ldc=m))
        keep.append((dA, dB, dC, O.dgemm(A, B, al, be, C)))
    h.dgemm_grouped(descs)
    torch.cuda.synchronize()
    h.check_device()
    for d, (_, _, dC, want) in zip(descs, keep):
        assert O.rel_errors(host(dC, (d["m"], d["n"])), want)[1] <= FRO_TOL


def test_summa_emulated(h):
    """SUMMA with every panel step as an INT8 Ozaki GEMM (8 slices)."""
    import torch

    M, N, K, b, p, q = 257, 131, 199, 32, 2, 3
    A, B, C = O.uniform((M, K), 1), O.uniform((K, N), 2), O.uniform((M, N), 3)
    o = O.orc()

    def pack(X, rows, cols):
        shapes = o.pblas_shapes(rows, cols, b, b, p, q)
        locs = [torch.zeros((max(c, 1), max(r, 1)), dtype=torch.float64, device="cuda") for r, c, _ in shapes]
        lld = [max(r, 1) for r, _, _ in shapes]
        dX = dev(X)
        h.pack_block_cyclic(rows, cols, b, b, p, q, ptr(dX), rows, [ptr(l) for l in locs], lld)
        return dX, locs, lld

    _, lA, lldA = pack(A, M, K)
    _, lB, lldB = pack(B, K, N)
    dC, lC, lldC = pack(C, M, N)
    h.summa(p, q, b, b, b, M, N, K, 1.5, [ptr(x) for x in lA], lldA, [ptr(x) for x in lB], lldB, -0.5,
            [ptr(x) for x in lC], lldC, mode=dgt.FP64_OZAKI_INT8, slices=8)
    h.unpack_block_cyclic(M, N, b, b, p, q, ptr(dC), M, [ptr(x) for x in lC], lldC)
    torch.cuda.synchronize()
    h.check_device()
    assert O.rel_errors(host(dC, (M, N)), O.dgemm(A, B, 1.5, -0.5, C))[1] <= FRO_TOL


@pytest.mark.parametrize("M,p,c", [(512, 4, 2), (384, 3, 1)])
def test_cannon_emulated(h, M, p, c):
    import torch

    A, B, C = O.uniform((M, M), 1), O.uniform((M, M), 2), O.uniform((M, M), 3)
    dA, dB, dC = dev(A), dev(B), dev(C)
    lm = M // p
    tiles = lambda: [torch.zeros((lm, lm), dtype=torch.float64, device="cuda") for _ in range(p * p)]
    tA, tB, tC = tiles(), tiles(), tiles()
    h.pack_cannon2d(M, p, ptr(dA), ptr(dB), ptr(dC), [ptr(x) for x in tA], [ptr(x) for x in tB],
                    [ptr(x) for x in tC])
    h.cannon25d(M, p, c, 1.0, [ptr(x) for x in tA], [ptr(x) for x in tB], 0.5, [ptr(x) for x in tC],
                mode=dgt.FP64_OZAKI_INT8, slices=8)
    h.unpack_cannon2d(M, p, ptr(dC), [ptr(x) for x in tC])
    torch.cuda.synchronize()
    h.check_device()
    assert O.rel_errors(host(dC, (M, M)), O.dgemm(A, B, 1.0, 0.5, C))[1] <= FRO_TOL


def test_grouped_emulated(h):
    import torch

    rng = np.random.default_rng(9)
    descs, keep = [], []
    for i in range(12):
        m, n, k = (int(x) for x in rng.integers(1, 400, 3))
        A, B, C = O.uniform((m, k), 500 + i), O.uniform((k, n), 600 + i), O.uniform((m, n), 700 + i)
        dA, dB, dC = dev(A), dev(B), dev(C)
        descs.append(dict(m=m, n=n, k=k, alpha=1.0, beta=-1.0, A=ptr(dA), lda=m, B=ptr(dB), ldb=k, C=ptr(dC), ldc=m))
        keep.append((dA, dB, dC, O.dgemm(A, B, 1.0, -1.0, C)))
    h.dgemm_grouped(descs, mode=dgt.FP64_OZAKI_INT8, slices=8)
    torch.cuda.synchronize()
    h.check_device()
    for d, (_, _, dC, want) in zip(descs, keep):
        assert O.rel_errors(host(dC, (d["m"], d["n"])), want)[1] <= FRO_TOL
