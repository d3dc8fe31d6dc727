"""FP64 emulation by CRT over INT8 residues (DGT_FP64_OZAKI2_INT8) through the C ABI:
bit for bit equal to the exact restatement (oracle.ozaki2_exact) for alpha = 1, beta = 0,
within relative Frobenius 1e-13 of the host FP64 GEMM otherwise (17 moduli: 58-bit
operands), identical across kernel variants, and the edge cases of the slice scheme."""
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


def run(h, ta, tb, m, n, k, alpha, beta, nmod, A, B, C):
    import torch

    dA, dB, dC = dev(A), dev(B), dev(C)
    h.dgemm(ta, tb, m, n, k, alpha, ptr(dA), A.shape[0], ptr(dB), B.shape[0], beta, ptr(dC), m,
            mode=dgt.FP64_OZAKI2_INT8, slices=nmod)
    torch.cuda.synchronize()
    h.check_device()
    return host(dC, (m, n))


def operands(ta, tb, m, n, k, seed, phi=None):
    ra, ca = (k, m) if ta == "T" else (m, k)
    rb, cb = (n, k) if tb == "T" else (k, n)
    gen = (lambda s, sd: O.ozaki_matrix(s, sd, phi)) if phi is not None else O.uniform
    return gen((ra, ca), seed), gen((rb, cb), seed + 1), O.uniform((m, n), seed + 2)


@pytest.mark.parametrize("ta,tb", [("N", "N"), ("N", "T"), ("T", "N"), ("T", "T")])
@pytest.mark.parametrize("shape", [(1, 1, 1), (7, 13, 5), (128, 256, 128), (130, 70, 333)])
def test_bitwise_equal_to_exact_restatement(h, ta, tb, shape):
    m, n, k = shape
    A, B, C = operands(ta, tb, m, n, k, sum(shape), phi=1.0)
    got = run(h, ta, tb, m, n, k, 1.0, 0.0, 17, A, B, C)
    assert np.array_equal(got, O.ozaki2_exact(A, B, 17, ta, tb))


@pytest.mark.parametrize("nmod", [8, 12, 14, 15, 16, 17, 18, 19, 20])
def test_bitwise_for_every_kernel_specialisation(h, nmod):
    """The reconstruction has modulus-count specialisations (14 to 20; three 41-bit FP64 limbs
    and a correctly rounded three-term sum up to 15 moduli, four 40-bit FP64 limbs with an
    integer rounding above) and generic kernels for the other counts: each equals the exact
    restatement bit for bit."""
    m, n, k = 97, 60, 300
    A, B, C = operands("N", "N", m, n, k, 50 + nmod, phi=1.0)
    got = run(h, "N", "N", m, n, k, 1.0, 0.0, nmod, A, B, C)
    assert np.array_equal(got, O.ozaki2_exact(A, B, nmod))


@pytest.mark.parametrize("nmod", [9, 14, 15, 16, 17, 20])
@pytest.mark.parametrize("scale", [-540, 0, 500])
def test_bitwise_across_the_exponent_range(h, nmod, scale):
    """Products that land in the subnormal range (~2^-1080), near 1 and near the overflow
    threshold (~2^1000), with a wide dynamic range inside each row: bit for bit the exact
    restatement (the exact integer product rounded once, then scaled) for every reconstruction
    form -- three FP64 limbs and a correctly rounded three-term sum up to 15 moduli, four FP64
    limbs with an integer rounding above, 32-bit integer limbs in the generic kernels."""
    m, n, k = 37, 29, 90
    A, B, _ = operands("N", "N", m, n, k, 70 + nmod, phi=2.0)
    A, B = np.ldexp(A, scale), np.ldexp(B, scale)
    got = run(h, "N", "N", m, n, k, 1.0, 0.0, nmod, A, B, np.zeros((m, n)))
    assert np.array_equal(got, O.ozaki2_exact(A, B, nmod))


@pytest.mark.parametrize("shape", [(300, 200, 1000), (513, 257, 4100)])
def test_alpha_beta_against_fp64(h, shape):
    m, n, k = shape
    A, B, C = operands("N", "N", m, n, k, 7)
    got = run(h, "N", "N", m, n, k, 1.5, -0.5, 17, A, B, C)
    assert O.rel_errors(got, O.dgemm(A, B, 1.5, -0.5, C))[1] <= FRO_TOL


def test_error_falls_with_moduli(h):
    m, n, k = 200, 150, 512
    A, B, C = operands("N", "N", m, n, k, 11, phi=0.5)
    want = O.dgemm(A, B)
    errs = [O.rel_errors(run(h, "N", "N", m, n, k, 1.0, 0.0, nm, A, B, C), want)[1] for nm in (10, 12, 14, 16, 17)]
    assert all(a > b for a, b in zip(errs, errs[1:]) if a > 1e-15)
    assert errs[-1] <= 1e-15  # the residual is the host FP64 GEMM's own rounding


@pytest.mark.parametrize("variant", [0, 1, 4, 5, 6, 7])
def test_kernel_variants_identical(variant):
    """Every residue-GEMM variant gives the same bits: 4 / 8 epilogue warps, the CTA pair, and
    (5, 6) the dynamic (tile, modulus) unit order, where clusters take units from an atomic
    counter; the second shape has ~40 units per cluster, so the order really varies."""
    for (m, n, k) in ((300, 520, 1000), (1100, 1500, 700)):
        A, B, C = operands("N", "N", m, n, k, 21)
        outs = []
        for v in (1, variant):
            with dgt.Handle() as hh:
                hh.set_tuning(dgt.TUNE_OZAKI_VARIANT, v)
                outs.append(run(hh, "N", "N", m, n, k, 1.25, 0.5, 17, A, B, C))
        assert np.array_equal(outs[0], outs[1]), (variant, m, n, k)


def test_nonfinite_and_zero_rows(h):
    m, n, k = 64, 48, 100
    A, B, C = operands("N", "N", m, n, k, 31)
    A[3, 7] = np.nan
    A[5, :] = 0.0
    B[2, 9] = np.inf
    got = run(h, "N", "N", m, n, k, 1.0, 0.0, 17, A, B, C)
    assert np.isnan(got[3, :]).all() and np.isnan(got[:, 9]).all()
    keep_r = [i for i in range(m) if i != 3]
    keep_c = [j for j in range(n) if j != 9]
    assert np.all(got[5, keep_c] == 0.0)
    want = O.dgemm(np.nan_to_num(A), np.nan_to_num(B, posinf=0.0))
    assert O.rel_errors(got[np.ix_(keep_r, keep_c)], want[np.ix_(keep_r, keep_c)])[1] <= FRO_TOL


def test_large_sampled(h):
    import torch

    n = 2048
    A, B = O.ozaki_matrix((n, n), 41, 0.5), O.ozaki_matrix((n, n), 42, 0.5)
    dA, dB, dC = dev(A), dev(B), torch.zeros((n, n), dtype=torch.float64, device="cuda")
    h.dgemm("N", "N", n, n, n, 1.0, ptr(dA), n, ptr(dB), n, 0.0, ptr(dC), n, mode=dgt.FP64_OZAKI2_INT8, slices=17)
    torch.cuda.synchronize()
    h.check_device()
    rows = np.random.default_rng(0).choice(n, 48, replace=False)
    got = host(dC, (n, n))[rows, :]
    assert O.rel_errors(got, A[rows, :] @ B)[1] <= 1e-15


def test_rejections(h):
    import torch

    x = torch.zeros(4, dtype=torch.float64, device="cuda")
    with pytest.raises(dgt.DgtError):  # modulus count outside [8, 20]
        h.dgemm("N", "N", 2, 2, 2, 1.0, ptr(x), 2, ptr(x), 2, 0.0, ptr(x), 2, mode=dgt.FP64_OZAKI2_INT8, slices=7)


def test_long_k_runs_in_chunks(h):
    """K = 150000 (beyond one exact INT32 residue product) runs as K-chunks of 65536."""
    import torch

    m, n, k = 3, 5, 150000
    A, B, C = O.uniform((m, k), 61), O.uniform((k, n), 62), O.uniform((m, n), 63)
    got = run(h, "N", "N", m, n, k, 1.5, -0.5, 17, A, B, C)
    assert O.rel_errors(got, O.dgemm(A, B, 1.5, -0.5, C))[1] <= FRO_TOL
    At, Bt = np.asfortranarray(A.T), np.asfortranarray(B.T)
    got_t = run(h, "T", "T", m, n, k, 1.5, -0.5, 17, At, Bt, C)
    assert O.rel_errors(got_t, O.dgemm(A, B, 1.5, -0.5, C))[1] <= FRO_TOL


@pytest.mark.parametrize("panels", [2, 3, 8])
@pytest.mark.parametrize("ta,tb", [("N", "N"), ("T", "T"), ("N", "T")])
def test_panels_change_nothing(h, panels, ta, tb):
    """op(B) in column panels (split and reconstruction on side streams beside the residue
    GEMM): the same result, bit for bit, as the product in one piece; ragged last panel."""
    m, n, k = 700, 1500, 900
    A, B, C = operands(ta, tb, m, n, k, 80 + panels, phi=1.0)
    h.set_tuning(dgt.TUNE_CRT_PANELS, 1)
    one = run(h, ta, tb, m, n, k, 1.5, -0.5, 14, A, B, C)
    h.set_tuning(dgt.TUNE_CRT_PANELS, panels)
    got = run(h, ta, tb, m, n, k, 1.5, -0.5, 14, A, B, C)
    h.set_tuning(dgt.TUNE_CRT_PANELS, 0)
    assert np.array_equal(got, one)
    assert O.rel_errors(got, O.dgemm(A, B, 1.5, -0.5, C, ta, tb))[1] <= FRO_TOL


def test_grouped_and_cannon_through_crt(h):
    import torch

    M, p, c = 512, 4, 2
    A, B, C = O.uniform((M, M), 1), O.uniform((M, M), 2), O.uniform((M, M), 3)
    dA, dB, dC = dev(A), dev(B), dev(C)
    lm = M // p
    tiles = lambda: [torch.zeros((lm, lm), dtype=torch.float64, device="cuda") for _ in range(p * p)]
    tA, tB, tC = tiles(), tiles(), tiles()
    h.pack_cannon2d(M, p, ptr(dA), ptr(dB), ptr(dC), [ptr(x) for x in tA], [ptr(x) for x in tB], [ptr(x) for x in tC])
    h.cannon25d(M, p, c, 1.0, [ptr(x) for x in tA], [ptr(x) for x in tB], 0.5, [ptr(x) for x in tC],
                mode=dgt.FP64_OZAKI2_INT8, slices=17)
    h.unpack_cannon2d(M, p, ptr(dC), [ptr(x) for x in tC])
    torch.cuda.synchronize()
    h.check_device()
    assert O.rel_errors(host(dC, (M, M)), O.dgemm(A, B, 1.0, 0.5, C))[1] <= FRO_TOL
