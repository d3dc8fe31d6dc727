"""Grouped FP64 emulation (INT8 Ozaki) through dgt_dgemm_grouped: every product of a batch
in one amax launch, one split launch and one persistent digit-GEMM launch.  The grouped pass
uses the same digits, flush groups and fold order as one Ozaki call per product, so its
results equal the per-product results bit for bit, and both are within relative Frobenius
1e-13 of the host FP64 GEMM."""
import numpy as np
import pytest

import dgt
import oracle as O
from devutil import dev, host, ptr

pytestmark = pytest.mark.gpu
FRO_TOL = 1e-13


def _operands(rng, m, n, k, ta, tb, seed):
    ra, ca = (k, m) if ta == "T" else (m, k)
    rb, cb = (n, k) if tb == "T" else (k, n)
    return O.uniform((ra, ca), seed), O.uniform((rb, cb), seed + 1), O.uniform((m, n), seed + 2)


def _batch(seed, count, lo, hi, mixed_trans=True):
    rng = np.random.default_rng(seed)
    items = []
    for i in range(count):
        m, n, k = (int(round(np.exp(rng.uniform(np.log(lo), np.log(hi))))) for _ in range(3))
        ta = "T" if (mixed_trans and rng.random() < 0.5) else "N"
        tb = "T" if (mixed_trans and rng.random() < 0.5) else "N"
        A, B, C = _operands(rng, m, n, k, ta, tb, 1000 * seed + 10 * i)
        alpha, beta = float(rng.uniform(-2, 2)), float(rng.uniform(-1, 1))
        items.append(dict(m=m, n=n, k=k, ta=ta, tb=tb, A=A, B=B, C=C, alpha=alpha, beta=beta))
    return items


def _descs(items):
    descs, keep = [], []
    for it in items:
        dA, dB, dC = dev(it["A"]), dev(it["B"]), dev(it["C"])
        keep.append((dA, dB, dC))
        descs.append(dict(m=it["m"], n=it["n"], k=it["k"], alpha=it["alpha"], beta=it["beta"], A=ptr(dA),
                          lda=it["A"].shape[0], B=ptr(dB), ldb=it["B"].shape[0], C=ptr(dC), ldc=it["m"],
                          transa=it["ta"], transb=it["tb"]))
    return descs, keep


def _want(it):
    return O.dgemm(it["A"], it["B"], it["alpha"], it["beta"], it["C"], it["ta"], it["tb"])


def test_grouped_matches_per_product_bitwise():
    """24 products, sizes log-uniform in [1, 700] plus a few with K up to 5000, mixed
    transposes: grouped == one Ozaki call per product, bit for bit."""
    import torch

    items = _batch(3, 20, 1, 700) + _batch(4, 4, 200, 5000)
    with dgt.Handle() as h:
        descs, keep = _descs(items)
        h.dgemm_grouped(descs, mode=dgt.FP64_OZAKI_INT8, slices=7)
        torch.cuda.synchronize()
        h.check_device()
        grouped = [host(k[2], (it["m"], it["n"])) for it, k in zip(items, keep)]
        for idx, (it, d) in enumerate(zip(items, descs)):
            dC = dev(it["C"])
            h.dgemm(it["ta"], it["tb"], it["m"], it["n"], it["k"], it["alpha"], d["A"], d["lda"], d["B"], d["ldb"],
                    it["beta"], ptr(dC), it["m"], mode=dgt.FP64_OZAKI_INT8, slices=7)
            torch.cuda.synchronize()
            single = host(dC, (it["m"], it["n"]))
            assert np.array_equal(single, grouped[idx]), (it["m"], it["n"], it["k"])
    for it, got in zip(items, grouped):
        assert O.rel_errors(got, _want(it))[1] <= FRO_TOL, (it["m"], it["n"], it["k"], it["ta"], it["tb"])


def test_grouped_is_three_kernel_launches():
    import torch

    items = _batch(5, 30, 16, 400, mixed_trans=False)
    with dgt.Handle() as h:
        descs, keep = _descs(items)
        n0 = h.launch_count()
        h.dgemm_grouped(descs, mode=dgt.FP64_OZAKI_INT8, slices=8)
        torch.cuda.synchronize()
        h.check_device()
        assert h.launch_count() - n0 == 3
    for it, k in zip(items, keep):
        assert O.rel_errors(host(k[2], (it["m"], it["n"])), _want(it))[1] <= FRO_TOL


def test_grouped_edge_products():
    """An empty product (m = 0), a product with K = 0 (C = beta * C), a 1 x 1 x 1 product and
    ordinary ones in the same grouped call."""
    import torch

    rng = np.random.default_rng(11)
    items = _batch(6, 5, 32, 300)
    items.append(dict(m=1, n=1, k=1, ta="N", tb="N", A=O.uniform((1, 1), 5), B=O.uniform((1, 1), 6),
                      C=O.uniform((1, 1), 7), alpha=1.5, beta=-0.5))
    items.append(dict(m=70, n=40, k=0, ta="N", tb="N", A=np.zeros((70, 1)), B=np.zeros((1, 40)),
                      C=O.uniform((70, 40), 8), alpha=1.0, beta=0.5))
    with dgt.Handle() as h:
        descs, keep = _descs(items)
        for d in descs:
            if d["k"] == 0:
                d["ldb"] = 1
        x = dev(np.zeros((1, 1)))
        descs.append(dict(m=0, n=5, k=5, alpha=1.0, beta=0.0, A=ptr(x), lda=1, B=ptr(x), ldb=5, C=ptr(x), ldc=1))
        h.dgemm_grouped(descs, mode=dgt.FP64_OZAKI_INT8, slices=8)
        torch.cuda.synchronize()
        h.check_device()
    for it, k in zip(items, keep):
        got = host(k[2], (it["m"], it["n"]))
        if it["k"] == 0:
            assert np.array_equal(got, 0.5 * it["C"])
        else:
            assert O.rel_errors(got, _want(it))[1] <= FRO_TOL


def test_grouped_ragged_batch_against_oracle():
    """96 products with M, N, K log-uniform in [128, 1536] (the shape law of the 256-product
    batching workload at a size the host oracle checks quickly)."""
    import torch

    items = _batch(7, 96, 128, 1536, mixed_trans=False)
    with dgt.Handle() as h:
        descs, keep = _descs(items)
        h.dgemm_grouped(descs, mode=dgt.FP64_OZAKI_INT8, slices=8)
        torch.cuda.synchronize()
        h.check_device()
    for it, k in zip(items, keep):
        assert O.rel_errors(host(k[2], (it["m"], it["n"])), _want(it))[1] <= FRO_TOL


@pytest.mark.parametrize("variant", [1, 6])
@pytest.mark.parametrize("nmod", [14, 16])
def test_grouped_crt_matches_per_product_bitwise(nmod, variant):
    """The CRT scheme in one grouped pass (amax, norm bounds, residue split, residue GEMM, reconstruction)
    equals one CRT call per product bit for bit: same operand bits per product, same residues,
    same exact reconstruction -- with the grouped GEMM's (tile, modulus) units in the static
    order (variant 1) and taken from the atomic counter (variant 6)."""
    import torch

    items = _batch(13, 20, 1, 700) + _batch(14, 4, 200, 5000)
    with dgt.Handle() as h:
        h.set_tuning(dgt.TUNE_OZAKI_VARIANT, variant)
        descs, keep = _descs(items)
        n0 = h.launch_count()
        h.dgemm_grouped(descs, mode=dgt.FP64_OZAKI2_INT8, slices=nmod)
        torch.cuda.synchronize()
        h.check_device()
        assert h.launch_count() - n0 == 5  # amax, norm bounds, residue split, GEMM, reconstruction
        grouped = [host(k[2], (it["m"], it["n"])) for it, k in zip(items, keep)]
        for idx, (it, d) in enumerate(zip(items, descs)):
            dC = dev(it["C"])
            h.dgemm(it["ta"], it["tb"], it["m"], it["n"], it["k"], it["alpha"], d["A"], d["lda"], d["B"], d["ldb"],
                    it["beta"], ptr(dC), it["m"], mode=dgt.FP64_OZAKI2_INT8, slices=nmod)
            torch.cuda.synchronize()
            assert np.array_equal(host(dC, (it["m"], it["n"])), grouped[idx]), (it["m"], it["n"], it["k"])
    for it, got in zip(items, grouped):
        assert O.rel_errors(got, _want(it))[1] <= FRO_TOL


def test_grouped_crt_edge_products():
    import torch

    items = _batch(15, 5, 32, 300)
    items.append(dict(m=1, n=1, k=1, ta="N", tb="N", A=O.uniform((1, 1), 5), B=O.uniform((1, 1), 6),
                      C=O.uniform((1, 1), 7), alpha=1.5, beta=-0.5))
    items.append(dict(m=70, n=40, k=0, ta="N", tb="N", A=np.zeros((70, 1)), B=np.zeros((1, 40)),
                      C=O.uniform((70, 40), 8), alpha=1.0, beta=0.5))
    with dgt.Handle() as h:
        descs, keep = _descs(items)
        for d in descs:
            if d["k"] == 0:
                d["ldb"] = 1
        x = dev(np.zeros((1, 1)))
        descs.append(dict(m=0, n=5, k=5, alpha=1.0, beta=0.0, A=ptr(x), lda=1, B=ptr(x), ldb=5, C=ptr(x), ldc=1))
        h.dgemm_grouped(descs, mode=dgt.FP64_OZAKI2_INT8, slices=17)
        torch.cuda.synchronize()
        h.check_device()
    for it, k in zip(items, keep):
        got = host(k[2], (it["m"], it["n"]))
        if it["k"] == 0:
            assert np.array_equal(got, 0.5 * it["C"])
        else:
            assert O.rel_errors(got, _want(it))[1] <= FRO_TOL
