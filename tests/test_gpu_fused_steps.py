"""Fused step schedules (DGT_TUNE_FUSE_STEPS, on by default) and dgt_cannon25d_batch.

Native 2.5D Cannon (Summa25Decomposer::multiply, src/25DCannon.cpp:286-375) reduces its
stacks (reduceResult, :203-228) inside its one persistent, cooperative launch: the partial
tiles come first in the tile order and count themselves, the stack-0 tiles add them once
counted.  The result is bit-identical to the step-by-step form (grouped launch, then a
stack-reduction launch), with one launch instead of two; with dgt_cannon25d_batch's extra
products in the same launch, both parts equal the Cannon multiply and dgt_dgemm_grouped run
apart, bit for bit.

CRT residues: each virtual rank is one product over all its k-blocks, and all ranks (and
stacks) run in one grouped pass of five launches.  A SUMMA result then equals the CRT product
of the whole matrices bit for bit (each C block is the product of its whole rows and columns,
scaled over the whole K, its residue sums exact); a Cannon tile equals the CRT products of its
stacks' concatenated k-blocks, added in stack order."""
import numpy as np
import pytest

import dgt
import oracle as O
from devutil import dev, host, ptr

pytestmark = pytest.mark.gpu
FRO_TOL = 1e-13


@pytest.fixture
def h():
    with dgt.Handle() as handle:
        yield handle


def _tiles(M, p, A, B, C, h):
    import torch

    lm = M // p
    mk = lambda: [torch.zeros((lm, lm), dtype=torch.float64, device="cuda") for _ in range(p * p)]
    tA, tB, tC = mk(), mk(), mk()
    dA, dB, dC = dev(A), dev(B), dev(C)
    h.pack_cannon2d(M, p, ptr(dA), ptr(dB), ptr(dC), [ptr(x) for x in tA], [ptr(x) for x in tB], [ptr(x) for x in tC])
    return tA, tB, tC


def _extras(count, seed, lo=16, hi=600):
    """Products with M, N, K log-uniform in [lo, hi], mixed transposes, alpha / beta."""
    import torch

    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        m, n, k = (int(round(np.exp(rng.uniform(np.log(lo), np.log(hi))))) for _ in range(3))
        ta, tb = rng.choice(["N", "T"]), rng.choice(["N", "T"])
        ra, ca = (k, m) if ta == "T" else (m, k)
        rb, cb = (n, k) if tb == "T" else (k, n)
        A, B, C = O.uniform((ra, ca), seed + 3 * i), O.uniform((rb, cb), seed + 3 * i + 1), O.uniform((m, n), seed + 3 * i + 2)
        out.append(dict(m=m, n=n, k=k, A=A, B=B, C=C, ta=str(ta), tb=str(tb), alpha=float(rng.uniform(0.5, 2)),
                        beta=float(rng.choice([0.0, -0.5]))))
    return out


def _descs(ex):
    bufs, descs = [], []
    for e in ex:
        dA, dB, dC = dev(e["A"]), dev(e["B"]), dev(e["C"])
        bufs.append((dA, dB, dC))
        descs.append(dict(m=e["m"], n=e["n"], k=e["k"], alpha=e["alpha"], beta=e["beta"], A=ptr(dA),
                          lda=e["A"].shape[0], B=ptr(dB), ldb=e["B"].shape[0], C=ptr(dC), ldc=e["m"],
                          transa=e["ta"], transb=e["tb"]))
    return bufs, descs


@pytest.mark.parametrize("M,p,c,beta", [(1024, 4, 2, -0.5), (1024, 4, 2, 0.0), (768, 4, 4, -0.5), (640, 2, 2, 0.0),
                                          (384, 4, 2, -0.5)])
def test_native_cannon_reduces_inside_its_launch(h, M, p, c, beta):
    import torch

    A, B, C = O.uniform((M, M), 1 + M), O.uniform((M, M), 2 + M), O.uniform((M, M), 3 + M)
    tA, tB, tC = _tiles(M, p, A, B, C, h)
    tE = [x.clone() for x in tC]
    pA, pB = [ptr(x) for x in tA], [ptr(x) for x in tB]
    torch.cuda.synchronize()
    n0 = h.launch_count()
    h.cannon25d(M, p, c, 1.5, pA, pB, beta, [ptr(x) for x in tC])
    n1 = h.launch_count()
    h.set_tuning(dgt.TUNE_FUSE_STEPS, 0)
    h.cannon25d(M, p, c, 1.5, pA, pB, beta, [ptr(x) for x in tE])
    n2 = h.launch_count()
    h.set_tuning(dgt.TUNE_FUSE_STEPS, 1)
    torch.cuda.synchronize()
    h.check_device()
    assert (n1 - n0, n2 - n1) == (1, 2)
    for r in range(p * p):
        assert torch.equal(tC[r], tE[r]), r
    dC = dev(np.zeros((M, M)))
    h.unpack_cannon2d(M, p, ptr(dC), [ptr(x) for x in tC])
    torch.cuda.synchronize()
    assert O.rel_errors(host(dC, (M, M)), O.dgemm(A, B, 1.5, beta, C))[1] <= FRO_TOL


@pytest.mark.parametrize("variant", [1, 10, 23, 25])
def test_native_batch_is_one_launch(h, variant):
    """Cannon 4 x 4 x 2 plus 40 ragged products in one launch: both parts bit for bit as run
    apart (the Cannon step-by-step, the products through dgt_dgemm_grouped)."""
    import torch

    M, p, c = 1024, 4, 2
    h.set_tuning(dgt.TUNE_DMMA_VARIANT, variant)
    A, B, C = O.uniform((M, M), 11), O.uniform((M, M), 12), O.uniform((M, M), 13)
    tA, tB, tC = _tiles(M, p, A, B, C, h)
    tE = [x.clone() for x in tC]
    pA, pB = [ptr(x) for x in tA], [ptr(x) for x in tB]
    ex = _extras(40, 100)
    bufs, descs = _descs(ex)
    bufs2, descs2 = _descs(ex)
    torch.cuda.synchronize()
    n0 = h.launch_count()
    h.cannon25d_batch(M, p, c, 1.0, pA, pB, 0.5, [ptr(x) for x in tC], descs)
    n1 = h.launch_count()
    h.set_tuning(dgt.TUNE_FUSE_STEPS, 0)
    h.cannon25d(M, p, c, 1.0, pA, pB, 0.5, [ptr(x) for x in tE])
    h.set_tuning(dgt.TUNE_FUSE_STEPS, 1)
    h.dgemm_grouped(descs2)
    torch.cuda.synchronize()
    h.check_device()
    assert n1 - n0 == 1
    for r in range(p * p):
        assert torch.equal(tC[r], tE[r]), r
    for e, b, b2 in zip(ex, bufs, bufs2):
        assert torch.equal(b[2], b2[2])
        got = host(b[2], (e["m"], e["n"]))
        want = O.dgemm(e["A"], e["B"], e["alpha"], e["beta"], e["C"], e["ta"], e["tb"])
        assert O.rel_errors(got, want)[1] <= FRO_TOL


def test_crt_summa_equals_whole_product(h):
    """SUMMA on a 3 x 2 grid with ragged blocks, CRT 14 moduli: each C block equals the CRT
    product of the whole matrices bit for bit, in one grouped pass (5 launches)."""
    import torch

    M, N, K, b, p, q = 1000, 700, 900, 96, 3, 2
    A, B, C = O.uniform((M, K), 21), O.uniform((K, N), 22), O.uniform((M, N), 23)
    o = O.orc()

    def pack(X, rows, cols):
        shapes = o.pblas_shapes(rows, cols, b, b, p, q)
        locs = [torch.zeros((max(cc, 1), max(r, 1)), dtype=torch.float64, device="cuda") for r, cc, _ in shapes]
        lld = [max(r, 1) for r, _, _ in shapes]
        dX = dev(X)
        h.pack_block_cyclic(rows, cols, b, b, p, q, ptr(dX), rows, [ptr(l) for l in locs], lld)
        return dX, locs, lld

    _, lA, lldA = pack(A, M, K)
    _, lB, lldB = pack(B, K, N)
    dC, lC, lldC = pack(C, M, N)
    torch.cuda.synchronize()
    n0 = h.launch_count()
    h.summa(p, q, b, b, b, M, N, K, 1.5, [ptr(x) for x in lA], lldA, [ptr(x) for x in lB], lldB, -0.5,
            [ptr(x) for x in lC], lldC, mode=dgt.FP64_OZAKI2_INT8, slices=14)
    n1 = h.launch_count()
    h.unpack_block_cyclic(M, N, b, b, p, q, ptr(dC), M, [ptr(x) for x in lC], lldC)
    dA, dB, dW = dev(A), dev(B), dev(C)
    h.dgemm("N", "N", M, N, K, 1.5, ptr(dA), M, ptr(dB), K, -0.5, ptr(dW), M, mode=dgt.FP64_OZAKI2_INT8, slices=14)
    torch.cuda.synchronize()
    h.check_device()
    assert n1 - n0 == 5
    got = host(dC, (M, N))
    assert np.array_equal(got, host(dW, (M, N)))
    assert O.rel_errors(got, O.dgemm(A, B, 1.5, -0.5, C))[1] <= FRO_TOL


@pytest.mark.parametrize("M,p,c,ta", [(512, 4, 2, "N"), (384, 2, 2, "T"), (768, 4, 4, "N")])
def test_crt_cannon_equals_stack_products(h, M, p, c, ta):
    """CRT Cannon in one grouped pass: tile (i, j) equals the CRT products of each stack's
    concatenated k-blocks (dgt_cannon_schedule's order), stack 0 with beta C, the further
    stacks added in order; 5 launches."""
    import torch

    lm, pc3 = M // p, p // c
    A, B, C = O.uniform((M, M), 31), O.uniform((M, M), 32), O.uniform((M, M), 33)
    tA, tB, tC = _tiles(M, p, A, B, C, h)
    C0 = [x.clone() for x in tC]
    torch.cuda.synchronize()
    n0 = h.launch_count()
    h.cannon25d(M, p, c, 1.25, [ptr(x) for x in tA], [ptr(x) for x in tB], 0.5, [ptr(x) for x in tC], ta=ta, tb="N",
                mode=dgt.FP64_OZAKI2_INT8, slices=14)
    n1 = h.launch_count()
    torch.cuda.synchronize()
    h.check_device()
    assert n1 - n0 == 5
    tiles_h = lambda ts: [x.cpu().numpy().T for x in ts]  # column-major lm x lm tiles
    hA, hB, hC0 = tiles_h(tA), tiles_h(tB), tiles_h(C0)
    for i in range(p):
        for j in range(p):
            acc = None
            for k in range(c):
                blocks, _ = dgt.cannon_schedule(p, c, i, j, k)
                assert len(blocks) == pc3
                # op(A) row panel and op(B) column panel over this stack's k-blocks
                if ta == "T":  # op(A) = A^T: the stored tiles A[t][i] hold op(A)'s (i, t) block transposed
                    Ar = np.vstack([hA[i * p + t] for t in blocks])  # (pc3 lm) x lm, stored as op(A)^T
                    lda, tA_ = pc3 * lm, "T"
                else:
                    Ar = np.hstack([hA[i * p + t] for t in blocks])  # lm x (pc3 lm)
                    lda, tA_ = lm, "N"
                Bc = np.vstack([hB[t * p + j] for t in blocks])
                dA, dB = dev(Ar), dev(Bc)
                dO = dev(hC0[i * p + j] if k == 0 else np.zeros((lm, lm)))
                h.dgemm(tA_, "N", lm, lm, pc3 * lm, 1.25, ptr(dA), lda, ptr(dB), pc3 * lm, 0.5 if k == 0 else 0.0,
                        ptr(dO), lm, mode=dgt.FP64_OZAKI2_INT8, slices=14)
                torch.cuda.synchronize()
                part = host(dO, (lm, lm))
                acc = part if acc is None else acc + part
            assert np.array_equal(tC[i * p + j].cpu().numpy().T, acc), (i, j)


def test_crt_batch_one_pass(h):
    """CRT Cannon 4 x 4 x 2 plus 24 ragged products in one grouped pass (5 launches): the
    Cannon tiles equal dgt_cannon25d's and the products dgt_dgemm_grouped's, bit for bit."""
    import torch

    M, p, c = 512, 4, 2
    A, B, C = O.uniform((M, M), 41), O.uniform((M, M), 42), O.uniform((M, M), 43)
    tA, tB, tC = _tiles(M, p, A, B, C, h)
    tE = [x.clone() for x in tC]
    pA, pB = [ptr(x) for x in tA], [ptr(x) for x in tB]
    ex = _extras(24, 300)
    bufs, descs = _descs(ex)
    bufs2, descs2 = _descs(ex)
    torch.cuda.synchronize()
    n0 = h.launch_count()
    h.cannon25d_batch(M, p, c, 1.0, pA, pB, 0.5, [ptr(x) for x in tC], descs, mode=dgt.FP64_OZAKI2_INT8, slices=15)
    n1 = h.launch_count()
    h.cannon25d(M, p, c, 1.0, pA, pB, 0.5, [ptr(x) for x in tE], mode=dgt.FP64_OZAKI2_INT8, slices=15)
    h.dgemm_grouped(descs2, mode=dgt.FP64_OZAKI2_INT8, slices=15)
    torch.cuda.synchronize()
    h.check_device()
    assert n1 - n0 == 5
    for r in range(p * p):
        assert torch.equal(tC[r], tE[r]), r
    for e, b, b2 in zip(ex, bufs, bufs2):
        assert torch.equal(b[2], b2[2])
        got = host(b[2], (e["m"], e["n"]))
        want = O.dgemm(e["A"], e["B"], e["alpha"], e["beta"], e["C"], e["ta"], e["tb"])
        assert O.rel_errors(got, want)[1] <= FRO_TOL
    dC = dev(np.zeros((M, M)))
    h.unpack_cannon2d(M, p, ptr(dC), [ptr(x) for x in tC])
    torch.cuda.synchronize()
    assert O.rel_errors(host(dC, (M, M)), O.dgemm(A, B, 1.0, 0.5, C))[1] <= FRO_TOL


def test_crt_steps_unfused_stay_within_tolerance(h):
    """The step-by-step CRT form (one grouped pass per step, stack reduction apart) is still
    there behind DGT_TUNE_FUSE_STEPS 0 and agrees with the FP64 product."""
    import torch

    M, p, c = 512, 4, 2
    A, B, C = O.uniform((M, M), 51), O.uniform((M, M), 52), O.uniform((M, M), 53)
    tA, tB, tC = _tiles(M, p, A, B, C, h)
    h.set_tuning(dgt.TUNE_FUSE_STEPS, 0)
    n0 = h.launch_count()
    h.cannon25d(M, p, c, 1.0, [ptr(x) for x in tA], [ptr(x) for x in tB], 0.5, [ptr(x) for x in tC],
                mode=dgt.FP64_OZAKI2_INT8, slices=15)
    n1 = h.launch_count()
    h.set_tuning(dgt.TUNE_FUSE_STEPS, 1)
    dC = dev(np.zeros((M, M)))
    h.unpack_cannon2d(M, p, ptr(dC), [ptr(x) for x in tC])
    torch.cuda.synchronize()
    h.check_device()
    assert n1 - n0 == 2 * 5 + 1
    assert O.rel_errors(host(dC, (M, M)), O.dgemm(A, B, 1.0, 0.5, C))[1] <= FRO_TOL
