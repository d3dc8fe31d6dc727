"""CPU pins of the CRT emulation's restatement (oracle.ozaki2_*): the residue/CRT identity
in exact integers, the operand-bit rule, and its accuracy against the host FP64 GEMM."""
import math

import numpy as np
import pytest

import oracle as O


@pytest.mark.parametrize("nmod,k", [(8, 5), (12, 64), (16, 300), (17, 40), (20, 128)])
def test_crt_identity_recovers_the_integer_product(nmod, k):
    A, B = O.uniform((6, k), nmod), O.ozaki_matrix((k, 5), nmod + 1, 2.0)
    X, exact = O.ozaki2_residue_check(A, B, nmod)
    assert (X == exact).all()


def test_norm_rule():
    """sigma_A + sigma_B: (2^sigma_A + sqrt(k)/2)(2^sigma_B + sqrt(k)/2) < (P/2)(1 - 2^-20), and one
    more bit breaks it (checked in integers, sqrt(k) bounded by isqrt)."""
    for nmod in range(8, 21):
        P = math.prod(O.OZAKI2_MODULI[:nmod])
        for k in (1, 7, 256, 4096, 16384, 65536):
            sa, sb = O.ozaki2_sigmas(nmod, k)
            assert sa - sb in (0, 1)
            hi = math.isqrt(k) + 1  # > sqrt(k)
            assert (2 ** (sa + 1) + hi) * (2 ** (sb + 1) + hi) * 2 ** 20 < 2 * P * (2 ** 20 - 1)
            s1 = sa + sb + 1
            lo = math.isqrt(k)  # <= sqrt(k)
            assert (2 ** ((s1 + 1) // 2 + 1) + lo) * (2 ** (s1 // 2 + 1) + lo) * 2 ** 20 >= 2 * P * (2 ** 20 - 1)
    assert all(math.gcd(p, q) == 1 for i, p in enumerate(O.OZAKI2_MODULI) for q in O.OZAKI2_MODULI[:i])


def test_row_scale_has_no_entry_cap():
    """A row with one large entry among small ones: its norm bound is the max itself, so the
    scaled entry reaches 2^sigma, beyond the FP64 mantissa (an integer already) while the
    small entries keep their bits down to 2^0; a dense row of equal entries is scaled by its
    norm."""
    k = 64
    single = np.full(k, 2.0 ** -30)
    single[5] = 0.75
    sg = O.ozaki2_sigmas(20, k)[0]
    s1 = O._row_scale(single, sg)
    big = abs(int(round(math.ldexp(0.75, s1))))
    assert 2 ** 76 <= big <= 2 ** sg and s1 == sg  # g = 0: 2^0 bounds the norm (about 0.75)
    assert int(round(math.ldexp(2.0 ** -30, s1))) == 2 ** (s1 - 30)  # small entries stay exact
    dense = np.full(k, 0.75)
    sg = O.ozaki2_sigmas(12, k)[0]
    s2 = O._row_scale(dense, sg)
    norm = math.sqrt(sum(math.ldexp(0.75, s2) ** 2 for _ in range(k)))
    assert norm <= 2 ** sg < 2 * norm * 2  # within a factor 2 of the bound (power-of-two scales)


def test_residue_split_arithmetic():
    """The kernels' integer split (ozaki2_split_residues, a restatement of its steps) gives the
    symmetric residue of rn(y) for every modulus: at the range edges (|y| up to 2^78, ties at
    .5, values next to 2^40 multiples) and on random magnitudes from 2^-3 to 2^78."""
    rng = np.random.default_rng(5)
    edges = []
    for e in (0, 1, 19, 20, 39, 40, 41, 52, 53, 59, 60, 61, 77):
        for d in (-1.0, -0.5, 0.0, 0.5, 1.0):
            edges += [2.0 ** e + d, -(2.0 ** e + d)]
    edges += [2.0 ** 78 - 2.0 ** 25, -(2.0 ** 78 - 2.0 ** 25), 0.5, -0.5, 1.5, -1.5, 2.5, -2.5, 0.0]
    mags = np.ldexp(rng.random(20000) + 0.5, rng.integers(-3, 78, 20000))
    y = np.concatenate([np.array(edges), mags * np.where(rng.random(20000) < 0.5, -1.0, 1.0)])
    assert np.all(np.abs(y) < 2.0 ** 78)
    exact = [int(round(float(v))) for v in y]  # rn, ties to even
    for p in O.OZAKI2_MODULI:
        got = O.ozaki2_split_residues(y, p)
        want = [((x + p // 2) % p) - p // 2 for x in exact]
        assert got.tolist() == want, p


def test_fp64_residue_path_gives_the_same_bytes():
    """The split's FP64 path (ozaki2_split_residues_fp64: exact t = yh c40 + yl, q = rint(t/p)
    by one FMA with fl(1/p), r = t - q p) writes the integer path's bytes for every modulus:
    non-integer y (the second rounding), exact ties of p = 256 (r = +-128, byte 0x80), and the
    range edges."""
    rng = np.random.default_rng(9)
    edges = []
    for e in (0, 1, 8, 39, 40, 41, 52, 53, 77):
        for d in (-1.0, -0.5, 0.0, 0.5, 1.0):
            edges += [2.0 ** e + d, -(2.0 ** e + d)]
    ties = [128.0 + 256.0 * j for j in range(-3, 4)] + [2.0 ** 40 * 3 + 128.0, -(2.0 ** 45) - 128.0]
    mags = np.ldexp(rng.random(300) + 0.5, rng.integers(-3, 78, 300))
    y = np.concatenate([np.array(edges + ties), mags * np.where(rng.random(300) < 0.5, -1.0, 1.0)])
    for p in O.OZAKI2_MODULI:
        assert O.ozaki2_split_residues_fp64(y, p).tolist() == O.ozaki2_split_residues(y, p).tolist(), p


def test_three_term_sum_is_correctly_rounded():
    """The reconstruction's final rounding (oracle.sum3_rn restates the kernel's steps): the
    sum d2 2^82 + d1 2^41 + d0 of three limb differences (integers below 2^53, overlapping)
    rounds once to nearest-even -- random limbs, heavy cancellation, and values an ulp around
    exact ties -- against exact rationals."""
    import random
    from fractions import Fraction

    rnd = random.Random(11)
    cases = []
    for i in range(6000):
        d0, d1 = rnd.randint(-2 ** 53 + 1, 2 ** 53 - 1), rnd.randint(-2 ** 53 + 1, 2 ** 53 - 1)
        d2 = rnd.randint(-2 ** 53 + 1, 2 ** 53 - 1) if i % 3 == 0 else rnd.randint(-2 ** 12, 2 ** 12)
        cases.append((d0, d1, d2))
    for i in range(3000):  # C = (odd K) 2^(s-1) + delta: one bit past the 53rd, ties and neighbours
        s_ = rnd.randint(54, 100)
        C = (2 * rnd.randint(2 ** 52, 2 ** 53 - 1) + 1) * 2 ** (s_ - 54) + rnd.choice([-1, 0, 1])
        C *= rnd.choice([-1, 1])
        d2, rem = divmod(C, 2 ** 82)
        d1, d0 = divmod(rem, 2 ** 41)
        t = rnd.randint(-2 ** 10, 2 ** 10)  # an overlapping split of the same value
        cases.append((d0 + t * 2 ** 41, d1 - t, d2))
    for d0, d1, d2 in cases:
        a, b, c = float(d2) * 2.0 ** 82, float(d1) * 2.0 ** 41, float(d0)
        assert (Fraction(a), Fraction(b), Fraction(c)) == (d2 * Fraction(2) ** 82, d1 * Fraction(2) ** 41, d0)
        assert O.sum3_rn(a, b, c) == float(Fraction(a) + Fraction(b) + Fraction(c)), (d0, d1, d2)


@pytest.mark.parametrize("nmod,limbs", [(14, 3), (15, 3), (16, 4), (18, 4), (20, 4)])
def test_limb_sums_with_integer_rounding(nmod, limbs):
    """The reconstruction's FP64-limb form with the integer rounding (oracle.crt_value_fi
    restates the kernel's steps) returns C' -- the symmetric residue of sum_j r_j W_j mod P --
    rounded once to nearest-even: random residues, and residues of values one bit past the
    53rd with ties and their neighbours, both signs, against Python's exact integers."""
    import random

    rnd = random.Random(100 + nmod)
    mods = O.OZAKI2_MODULI[:nmod]
    P = math.prod(mods)
    targets = []
    for _ in range(150):
        r = [rnd.randrange(p) for p in mods]
        x = sum(ri * (P // p) * pow((P // p) % p, -1, p) for ri, p in zip(r, mods)) % P
        targets.append(x - P if x > P // 2 else x)
    for _ in range(150):
        s_ = rnd.randint(54, int(math.log2(P)) - 3)
        C = (2 * rnd.randint(2 ** 52, 2 ** 53 - 1) + 1) * 2 ** (s_ - 54) + rnd.choice([-1, 0, 1])
        targets.append(C * rnd.choice([-1, 1]))
    targets += [0, 1, -1, 2 ** 53 + 1, -(2 ** 53 + 1)]
    for C in targets:
        res = [C % p for p in mods]
        assert O.crt_value_fi(res, nmod, limbs) == float(C), (nmod, C)


def _exact_max_scaled(A, B, nmod):
    """The same integer emulation with every row / column scaled by its max instead (the
    bound k 2^(2 beta) < P/2): the reference point the norm scaling improves on."""
    m, k = A.shape
    n = B.shape[1]
    lg = sum(math.log2(p) for p in O.OZAKI2_MODULI[:nmod])
    beta = math.floor((lg - 1 - math.log2(k)) / 2 - 1e-9)
    ea = [math.frexp(float(np.max(np.abs(A[i]))))[1] for i in range(m)]
    fb = [math.frexp(float(np.max(np.abs(B[:, j]))))[1] for j in range(n)]
    Ai = [[int(round(math.ldexp(float(A[i, t]), beta - ea[i]))) for t in range(k)] for i in range(m)]
    Bi = [[int(round(math.ldexp(float(B[t, j]), beta - fb[j]))) for t in range(k)] for j in range(n)]
    C = np.empty((m, n))
    for i in range(m):
        for j in range(n):
            C[i, j] = math.ldexp(float(sum(x * y for x, y in zip(Ai[i], Bi[j]))), ea[i] + fb[j] - 2 * beta)
    return C


@pytest.mark.parametrize("phi", [0.5, 2.0])
def test_norm_scaling_beats_max_scaling(phi):
    """Entries (U - 0.5) exp(phi N(0,1)): a row's 2-norm is far below sqrt(k) times its max, so
    scaling by the norm keeps more bits: at 12 moduli both errors are several times smaller."""
    A, B = O.ozaki_matrix((20, 400), 21, phi), O.ozaki_matrix((400, 16), 22, phi)
    want = O.dgemm(A, B)
    norm = O.rel_errors(O.ozaki2_exact(A, B, 12), want)
    mx = O.rel_errors(_exact_max_scaled(A, B, 12), want)
    assert norm[1] < mx[1] / 3 and norm[0] < mx[0]


def test_rows_at_the_norm_bound():
    """Dense rows whose scaled entries round up: the CRT identity still holds."""
    k = 64
    A = np.full((3, k), 1.0 - 2.0 ** -60)
    A[1] *= -1.0
    B = O.uniform((k, 4), 9)
    X, exact = O.ozaki2_residue_check(A, B, 12)
    assert (X == exact).all()


def test_exact_restatement_accuracy():
    A, B = O.ozaki_matrix((40, 300), 3, 0.5), O.ozaki_matrix((300, 30), 4, 0.5)
    want = O.dgemm(A, B)
    assert O.rel_errors(O.ozaki2_exact(A, B, 17), want)[1] <= 1e-15
    assert O.rel_errors(O.ozaki2_exact(A, B, 12), want)[1] > 1e-14  # fewer moduli, fewer bits
