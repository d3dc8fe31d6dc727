"""Pack / unpack kernels through the C ABI, bit-exact against the oracle (which is
itself pinned to the reference's own code: tests/test_oracle.py)."""
import os

import numpy as np
import pytest

import dgt
import oracle as O
from devutil import dev, host, ptr

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def h():
    with dgt.Handle() as handle:
        yield handle


def _cyclic_roundtrip(h, M, N, mb, nb, p, q, seed, G=None):
    import torch

    G = O.uniform((M, N), seed) if G is None else G
    want = O.orc().pblas_scatter(G, mb, nb, p, q)
    dG = dev(G)
    locs = [torch.full((max(w.shape[1], 1), max(w.shape[0], 1)), -7.0, dtype=torch.float64, device="cuda")
            for w in want]
    lld = [max(w.shape[0], 1) for w in want]
    h.pack_block_cyclic(M, N, mb, nb, p, q, ptr(dG), M, [ptr(l) for l in locs], lld)
    torch.cuda.synchronize()
    for l, w in zip(locs, want):
        assert np.array_equal(host(l, (max(w.shape[0], 1), max(w.shape[1], 1)))[:w.shape[0], :w.shape[1]], w)
    dG2 = torch.zeros_like(dG)
    h.unpack_block_cyclic(M, N, mb, nb, p, q, ptr(dG2), M, [ptr(l) for l in locs], lld)
    torch.cuda.synchronize()
    assert torch.equal(dG, dG2)


def test_block_cyclic_golden_cases(h):
    g = np.load(os.path.join(GOLD, "pblas.npz"))
    idx = 0
    while f"pblas{idx}_params" in g:
        M, N, Mb, Nb, p, q = (int(v) for v in g[f"pblas{idx}_params"])
        _cyclic_roundtrip(h, M, N, Mb, Nb, p, q, 0, G=g[f"pblas{idx}_global"])
        idx += 1


@pytest.mark.parametrize("case", [(1, 1, 1, 1, 1, 1), (5, 3, 1, 1, 2, 3), (1023, 777, 64, 32, 3, 5),
                                  (4096, 4096, 512, 512, 2, 2)])
def test_block_cyclic_shapes(h, case):
    _cyclic_roundtrip(h, *case, seed=5)


@pytest.mark.parametrize("name,M,N", [("A", 15000, 9000), ("B", 9000, 17000), ("C", 15000, 17000)])
def test_block_cyclic_config2_full_size(h, name, M, N):
    """All three matrices of the ragged SUMMA configuration (M = 15000, N = 17000, K = 9000) on
    a 4 x 4 grid with 256 blocks, packed and unpacked at full size: bit-exact vs the oracle."""
    _cyclic_roundtrip(h, M, N, 256, 256, 4, 4, seed={"A": 42, "B": 43, "C": 44}[name])


def test_block_cyclic_rejects_bad_lld(h):
    with pytest.raises(dgt.DgtError) as e:
        h.pack_block_cyclic(100, 100, 10, 10, 2, 2, 1, 100, [1, 1, 1, 1], [10, 50, 50, 50])
    assert e.value.status == dgt.INVALID_VALUE


@pytest.mark.parametrize("M,N,K,P", [(10, 12, 7, 4), (13, 11, 5, 6), (20, 20, 20, 2), (333, 171, 80, 5),
                                     (1000, 900, 64, 16)])
@pytest.mark.parametrize("cm", [True, False])
def test_block2d(h, M, N, K, P, cm):
    import torch

    A, B, C = O.uniform((M, K), 1), O.uniform((K, N), 2), O.uniform((M, N), 3)
    lA, lB, lC = O.orc().block2d_deliver(A, B, C, P, cm)
    order = "F" if cm else "C"

    def d(x):  # device buffer holding x's bytes in the given order
        return torch.from_numpy(np.ascontiguousarray(np.asarray(x, order=order).ravel(order=order))).cuda()

    dA, dB, dC = d(A), d(B), d(C)
    oA = [torch.zeros(x.size, dtype=torch.float64, device="cuda") for x in lA]
    oB = [torch.zeros(x.size, dtype=torch.float64, device="cuda") for x in lB]
    oC = [torch.zeros(x.size, dtype=torch.float64, device="cuda") for x in lC]
    h.pack_block2d(M, N, K, P, cm, ptr(dA), ptr(dB), ptr(dC), [ptr(x) for x in oA], [ptr(x) for x in oB],
                   [ptr(x) for x in oC])
    torch.cuda.synchronize()
    for got, want in ((oA, lA), (oB, lB), (oC, lC)):
        for x, w in zip(got, want):
            assert np.array_equal(x.cpu().numpy(), np.asarray(w, order=order).ravel(order=order))
    dC2 = torch.zeros_like(dC)
    h.unpack_block2d(M, N, P, cm, ptr(dC2), [ptr(x) for x in oC])
    torch.cuda.synchronize()
    # the product's gather is the intended strided copy: it always restores C (the
    # reference's copyBlock shortcut does not for P=2, M==N, column-major)
    assert torch.equal(dC2, dC)


@pytest.mark.parametrize("M,p", [(8, 2), (16, 4), (300, 3), (4096, 4)])
def test_cannon_pack_unpack(h, M, p):
    import torch

    A, B, C = O.uniform((M, M), 1), O.uniform((M, M), 2), O.uniform((M, M), 3)
    lA, lB, lC = O.orc().cannon_decompose(A, B, C, p)
    dA, dB, dC = dev(A), dev(B), dev(C)
    lm = M // p
    oA = [torch.zeros((lm, lm), dtype=torch.float64, device="cuda") for _ in range(p * p)]
    oB = [torch.zeros_like(x) for x in oA]
    oC = [torch.zeros_like(x) for x in oA]
    h.pack_cannon2d(M, p, ptr(dA), ptr(dB), ptr(dC), [ptr(x) for x in oA], [ptr(x) for x in oB],
                    [ptr(x) for x in oC])
    torch.cuda.synchronize()
    for got, want in ((oA, lA), (oB, lB), (oC, lC)):
        for x, w in zip(got, want):
            assert np.array_equal(host(x, (lm, lm)), w)
    dC2 = torch.zeros_like(dC)
    h.unpack_cannon2d(M, p, ptr(dC2), [ptr(x) for x in oC])
    torch.cuda.synchronize()
    assert torch.equal(dC2, dC)


@pytest.mark.parametrize("rows,cols,ldS,ldD,cm", [(5, 7, 9, 6, True), (64, 3, 64, 64, True), (3, 64, 70, 65, False),
                                                  (1, 1, 1, 1, True)])
def test_copy_block(h, rows, cols, ldS, ldD, cm):
    import torch

    r, c = (rows, cols) if cm else (cols, rows)
    src = np.random.default_rng(0).standard_normal(ldS * c)
    dst0 = np.random.default_rng(1).standard_normal(ldD * c)
    ds, dd = torch.from_numpy(src).cuda(), torch.from_numpy(dst0.copy()).cuda()
    h.copy_block(rows, cols, ptr(ds), ptr(dd), ldS, ldD, cm)
    torch.cuda.synchronize()
    want = dst0.copy()
    for j in range(c):
        want[j * ldD:j * ldD + r] = src[j * ldS:j * ldS + r]
    assert np.array_equal(dd.cpu().numpy(), want)

