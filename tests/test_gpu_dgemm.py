"""Native FP64 DMMA GEMM through the C ABI vs the host FP64 GEMM oracle (OpenBLAS).

Tolerance: relative Frobenius error <= 1e-13 (the FP64 acceptance bound for the plain
method), max elementwise relative error reported."""
import numpy as np
import pytest

import dgt
import oracle as O
from devutil import dev, host, ptr

pytestmark = pytest.mark.gpu
FRO_TOL = 1e-13


@pytest.fixture(scope="module")
def h():
    with dgt.Handle() as handle:
        yield handle


def run(h, ta, tb, m, n, k, alpha, beta, seed=0, pad=(0, 0, 0), offset=0):
    import torch

    ra, ca = (k, m) if ta == "T" else (m, k)
    rb, cb = (n, k) if tb == "T" else (k, n)
    lda, ldb, ldc = ra + pad[0], rb + pad[1], m + pad[2]
    A = O.uniform((lda, ca), seed + 1)
    B = O.uniform((ldb, cb), seed + 2)
    C = O.uniform((ldc, n), seed + 3)
    dA, dB, dC = dev(A), dev(B), dev(C)
    # offset shifts the operand base by whole elements (misaligned-to-16B path)
    h.dgemm(ta, tb, m, n, k, alpha, ptr(dA) + 8 * offset, lda, ptr(dB) + 8 * offset, ldb, beta, ptr(dC), ldc)
    torch.cuda.synchronize()
    h.check_device()
    got = host(dC, (ldc, n))
    # the operand the kernel sees starts `offset` elements in; the element past the end of
    # the flat buffer only ever lands in a padding row, so pad the host view with a zero
    fa = np.concatenate([A.ravel(order="F")[offset:], np.zeros(offset)])
    fb = np.concatenate([B.ravel(order="F")[offset:], np.zeros(offset)])
    Aop = fa.reshape((lda, ca), order="F")[:ra, :]
    Bop = fb.reshape((ldb, cb), order="F")[:rb, :]
    want = O.dgemm(Aop, Bop, alpha, beta, C[:m, :], ta, tb)
    assert np.array_equal(got[m:, :], C[m:, :]), "rows beyond m were written"
    return O.rel_errors(got[:m, :], want)


@pytest.mark.parametrize("ta,tb", [("N", "N"), ("N", "T"), ("T", "N"), ("T", "T")])
@pytest.mark.parametrize("shape", [(128, 128, 16), (257, 193, 131), (1, 1, 1), (7, 13, 5), (300, 64, 1000)])
def test_dgemm_ops_and_ragged_shapes(h, ta, tb, shape):
    m, n, k = shape
    _, fro = run(h, ta, tb, m, n, k, 1.5, -0.5)
    assert fro <= FRO_TOL


def test_dgemm_padded_leading_dims_and_misaligned_base(h):
    _, fro = run(h, "N", "N", 200, 150, 90, 1.0, 1.0, pad=(3, 5, 7))
    assert fro <= FRO_TOL
    _, fro = run(h, "N", "T", 129, 131, 77, 2.0, 0.0, pad=(1, 1, 1), offset=1)
    assert fro <= FRO_TOL


def test_beta_zero_does_not_read_c(h):
    import torch

    m, n, k = 64, 48, 32
    A, B = O.uniform((m, k), 5), O.uniform((k, n), 6)
    C = np.full((m, n), np.nan, order="F")
    dA, dB, dC = dev(A), dev(B), dev(C)
    h.dgemm("N", "N", m, n, k, 1.0, ptr(dA), m, ptr(dB), k, 0.0, ptr(dC), m)
    torch.cuda.synchronize()
    got = host(dC, (m, n))
    assert np.isfinite(got).all()
    assert O.rel_errors(got, A @ B)[1] <= FRO_TOL


def test_k_zero_scales_c(h):
    import torch

    m, n = 33, 17
    C = O.uniform((m, n), 9)
    dC = dev(C)
    dummy = dev(np.zeros((1, 1)))
    h.dgemm("N", "N", m, n, 0, 3.0, ptr(dummy), m, ptr(dummy), 1, 2.0, ptr(dC), m)
    torch.cuda.synchronize()
    assert np.array_equal(host(dC, (m, n)), 2.0 * C)


def test_invalid_arguments_return_status(h):
    with pytest.raises(dgt.DgtError) as e:
        h.dgemm("X", "N", 4, 4, 4, 1.0, 1, 4, 1, 4, 0.0, 1, 4)
    assert e.value.status == dgt.INVALID_VALUE
    with pytest.raises(dgt.DgtError) as e:
        h.dgemm("N", "N", 4, 4, 4, 1.0, 1, 3, 1, 4, 0.0, 1, 4)  # lda < m
    assert e.value.status == dgt.INVALID_VALUE
    with pytest.raises(dgt.DgtError) as e:
        h.dgemm("N", "N", -1, 4, 4, 1.0, 1, 4, 1, 4, 0.0, 1, 4)
    assert e.value.status == dgt.INVALID_VALUE


def test_config1_dgemm_4096(h):
    """M = N = K = 4096, alpha = 1, beta = 0, U[-1,1): Frobenius <= 1e-13 vs host dgemm."""
    import torch

    n = 4096
    A, B = O.uniform((n, n), 20261203), O.uniform((n, n), 20261204)
    dA, dB = dev(A), dev(B)
    dC = torch.full((n, n), float("nan"), dtype=torch.float64, device="cuda")
    h.dgemm("N", "N", n, n, n, 1.0, ptr(dA), n, ptr(dB), n, 0.0, ptr(dC), n)
    torch.cuda.synchronize()
    mx, fro = O.rel_errors(host(dC, (n, n)), A @ B)
    assert fro <= FRO_TOL, (mx, fro)


def test_double_double_sample_error(h):
    """The GPU result is as close to the exactly rounded product as host OpenBLAS is."""
    import torch

    m, n, k = 512, 512, 2048
    A, B = O.uniform((m, k), 31), O.uniform((k, n), 32)
    dA, dB = dev(A), dev(B)
    dC = torch.zeros((n, m), dtype=torch.float64, device="cuda")
    h.dgemm("N", "N", m, n, k, 1.0, ptr(dA), m, ptr(dB), k, 0.0, ptr(dC), m)
    torch.cuda.synchronize()
    got = host(dC, (m, n))
    rng = np.random.default_rng(0)
    rows, cols = rng.integers(0, m, 400), rng.integers(0, n, 400)
    exact = O.orc().dgemm_dd_sample(A, B, 1.0, 0.0, None, rows, cols)
    gpu_err = np.abs(got[rows, cols] - exact) / np.abs(exact)
    cpu_err = np.abs((A @ B)[rows, cols] - exact) / np.abs(exact)
    assert np.median(gpu_err) <= 4 * max(np.median(cpu_err), 1e-17)


@pytest.mark.parametrize("variant", list(range(26)))
def test_dmma_kernel_variants(variant):
    """Every tuning variant of the native kernel (DMMA shape m16n8k4/k8/k16, K depth, ring
    depth, 8 or 16 warps, 64- or 128-bit fragment loads) on ragged shapes, all four
    transpose pairs, padded and 16-byte-misaligned operands."""
    with dgt.Handle() as hh:
        hh.set_tuning(dgt.TUNE_DMMA_VARIANT, variant)
        for ta, tb in (("N", "N"), ("N", "T"), ("T", "N"), ("T", "T")):
            _, fro = run(hh, ta, tb, 257, 193, 131, 1.5, -0.5, seed=variant)
            assert fro <= FRO_TOL, (variant, ta, tb)
        _, fro = run(hh, "N", "N", 300, 64, 1000, 1.0, 0.0, seed=variant)
        assert fro <= FRO_TOL
        _, fro = run(hh, "N", "T", 129, 131, 77, 2.0, 1.0, pad=(1, 1, 1), offset=1)
        assert fro <= FRO_TOL


def _raw(h, ta, tb, m, n, k, alpha, beta, A, B, C, lda, ldb):
    import torch

    dA, dB, dC = dev(A), dev(B), dev(C)
    h.dgemm(ta, tb, m, n, k, alpha, ptr(dA), lda, ptr(dB), ldb, beta, ptr(dC), m)
    torch.cuda.synchronize()
    h.check_device()
    return host(dC, (m, n))


@pytest.mark.parametrize("tma,base", [(14, 2), (15, 1), (16, 7), (17, 1), (18, 2), (19, 1), (20, 7), (21, 2), (22, 2)])
def test_tma_variants_bit_identical_to_cp_async(tma, base):
    """Variants 14-22 bring the operand tiles in by TMA (bulk-tensor loads completing on an
    mbarrier per stage; 18-22 release stages through per-stage empty barriers instead of a CTA
    barrier per k-tile) into the same padded shared-memory layout the cp.async loader writes,
    so with the same DMMA shape and K depth the result is bit for bit the cp.async kernel's:
    ragged edges (zero-filled out-of-range boxes), all four transpose pairs, beta != 0, a K
    that is not a multiple of the stage depth, and a problem spanning several waves of tiles."""
    for (m, n, k), (ta, tb) in (((513, 385, 300), ("N", "N")), ((513, 385, 300), ("N", "T")),
                                ((513, 385, 300), ("T", "N")), ((513, 385, 300), ("T", "T")),
                                ((256, 256, 64), ("N", "N")), ((2304, 2048, 1000), ("N", "N"))):
        ra, ca = (k, m) if ta == "T" else (m, k)
        rb, cb = (n, k) if tb == "T" else (k, n)
        A, B, C = O.uniform((ra, ca), m + 1), O.uniform((rb, cb), n + 2), O.uniform((m, n), k + 3)
        out = {}
        for v in (tma, base):
            with dgt.Handle() as hh:
                hh.set_tuning(dgt.TUNE_DMMA_VARIANT, v)
                out[v] = _raw(hh, ta, tb, m, n, k, 1.5, -0.5, A, B, C, ra, rb)
        assert np.array_equal(out[tma], out[base]), (tma, m, n, k, ta, tb)
        assert O.rel_errors(out[tma], O.dgemm(A, B, 1.5, -0.5, C, ta, tb))[1] <= FRO_TOL



@pytest.mark.parametrize("dec,base", [(23, 2), (24, 1), (25, 17)])
def test_grouped_dec_variants_bit_identical(dec, base):
    """Variants 23-25 run the grouped kernel without CTA barriers in its main loop (stages
    signalled by cp.async mbarrier arrivals, released per warp, the load cursor running across
    tiles and problems): bit for bit the barrier kernel of the same shape, on 48 ragged grouped
    products (transposes, misaligned operands, K = 0, a one-element product, several waves),
    and against host FP64."""
    import torch

    rng = np.random.default_rng(dec)
    specs = []
    for i in range(48):
        m, n, k = (int(x) for x in rng.integers(1, 700, 3))
        if i == 0:
            m, n, k = 1, 1, 1
        if i == 1:
            k = 0
        ta, tb = str(rng.choice(["N", "T"])), str(rng.choice(["N", "T"]))
        ra, ca = (k, m) if ta == "T" else (m, k)
        rb, cb = (n, k) if tb == "T" else (k, n)
        specs.append((m, n, k, ta, tb, O.uniform((max(ra, 1), max(ca, 1)), 3 * i + 1),
                      O.uniform((max(rb, 1), max(cb, 1)), 3 * i + 2), O.uniform((m, n), 3 * i + 3)))
    outs = {}
    for v in (dec, base):
        keep, descs = [], []
        for m, n, k, ta, tb, A, B, C in specs:
            dA, dB, dC = dev(A), dev(B), dev(C)
            keep.append((dA, dB, dC))
            descs.append(dict(m=m, n=n, k=k, alpha=1.25, beta=-0.5, A=ptr(dA), lda=A.shape[0], B=ptr(dB),
                              ldb=B.shape[0], C=ptr(dC), ldc=m, transa=ta, transb=tb))
        with dgt.Handle() as hh:
            hh.set_tuning(dgt.TUNE_DMMA_VARIANT, v)
            hh.dgemm_grouped(descs)
            torch.cuda.synchronize()
            hh.check_device()
        outs[v] = [host(x[2], (sp[0], sp[1])) for x, sp in zip(keep, specs)]
    for i, (m, n, k, ta, tb, A, B, C) in enumerate(specs):
        assert np.array_equal(outs[dec][i], outs[base][i]), i
        want = O.dgemm(A[:, :k] if ta == "N" else A[:k, :], B[:k, :] if tb == "N" else B[:, :k], 1.25, -0.5, C,
                       ta, tb) if k > 0 else -0.5 * C
        assert O.rel_errors(outs[dec][i], want)[1] <= FRO_TOL, i
