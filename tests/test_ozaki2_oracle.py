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


def test_operand_bits_rule():
    for nmod in range(8, 21):
        P = math.prod(O.OZAKI2_MODULI[:nmod])
        for k in (1, 7, 256, 4096, 16384, 65536):
            b = O.ozaki2_beta(nmod, k)
            if b < 1:
                continue
            assert 2 * k * 2 ** (2 * b) < P  # operands are rounded to nearest: |A'|, |B'| <= 2^beta
            assert b == 58 or 2 * k * (2 ** (b + 1) - 1) ** 2 >= P // 2  # within a bit of the largest
    assert O.ozaki2_beta(17, 16384) == 58 and O.ozaki2_beta(16, 16384) == 55
    assert all(math.gcd(p, q) == 1 for i, p in enumerate(O.OZAKI2_MODULI) for q in O.OZAKI2_MODULI[:i])


def test_rounded_operands_reach_the_bound():
    """A row whose max rounds up gives |A'| = 2^beta exactly; the CRT identity still holds."""
    k = 64
    A = np.full((3, k), 1.0 - 2.0 ** -60)  # just below 2^0: scaled to 2^beta - 2^(beta-60), rounds to 2^beta
    A[1] *= -1.0
    B = O.uniform((k, 4), 9)
    X, exact = O.ozaki2_residue_check(A, B, 12)
    assert (X == exact).all()
    beta = O.ozaki2_beta(12, k)
    assert abs(int(round(math.ldexp(A[0, 0], beta - 0)))) == 2 ** beta


def test_exact_restatement_accuracy():
    A, B = O.ozaki_matrix((40, 300), 3, 0.5), O.ozaki_matrix((300, 30), 4, 0.5)
    want = O.dgemm(A, B)
    assert O.rel_errors(O.ozaki2_exact(A, B, 17), want)[1] <= 1e-15
    assert O.rel_errors(O.ozaki2_exact(A, B, 12), want)[1] > 1e-13  # fewer moduli, fewer bits
