"""The reference's exact MpFloat Cholesky (xpotrf, algebra/dense/blas/mpfr.rs:726-789) on the GPU.

sdpxg_mp_potrf must return the oracle's bits (oracle/exact.py xpotrf: exact dots rounded once,
differences, square roots and divisions correctly rounded) on symmetric diagonally dominant
matrices from the reference's test generator, at 64 to 512 bits, lower and upper storage, and
the LAPACK-style info (j + 1) at the first non-positive pivot.  The square root's rounding is
pinned against mpmath on the CPU.
"""
from fractions import Fraction
import sys
from pathlib import Path

import pytest

from oracle import exact as X

sys.path.insert(0, str(Path(__file__).resolve().parent / "golden"))
import make_ldl_fixtures as F  # noqa: E402  (the generator of symmetric test matrices)

CASES = [(1, 9, "L", 4, 41), (2, 20, "L", 8, 42), (4, 37, "U", 6, 43), (8, 12, "L", 3, 44), (4, 64, "U", 4, 45)]


def test_oracle_sqrt_matches_mpmath():
    mpmath = pytest.importorskip("mpmath")
    rng = X.Lcg(3)
    for n in (1, 2, 4, 8):
        for v in X.random_values(n, rng, 100, 30):
            if v.is_zero():
                continue
            v.neg = False
            r = X.mp_sqrt(n, v)
            with mpmath.workprec(64 * n):
                ref = mpmath.sqrt(mpmath.mpf(v.mant) * mpmath.mpf(2) ** (v.exp - v.p))
            _, man, e2, _ = ref._mpf_
            assert r.fraction() == Fraction(int(man)) * Fraction(2) ** int(e2)


@pytest.mark.gpu
@pytest.mark.parametrize("limbs,n,uplo,spread,seed", CASES)
def test_mp_potrf_bitwise(limbs, n, uplo, spread, seed):
    from sdpx_b200.solver import KernelContext
    A = F.matrix(limbs, n, spread, seed)
    expect = list(A)
    info = X.xpotrf(limbs, uplo, n, expect, n)
    assert info == 0
    raw, ginfo, st = KernelContext().mp_potrf(limbs, uplo, n, X.pack_array(A), n)
    assert ginfo == 0 and st == 0
    got = X.unpack_array(limbs, raw)
    bad = [(i % n, i // n) for i in range(n * n) if not got[i] == expect[i]]
    assert not bad, bad[:5]


@pytest.mark.gpu
def test_mp_potrf_reports_first_nonpositive_pivot():
    from sdpx_b200.solver import KernelContext
    limbs, n = 4, 16
    A = F.matrix(limbs, n, 4, 46)
    A[5 + 5 * n] = X.from_fraction(limbs, Fraction(-1))  # pivot 5 negative
    expect = list(A)
    info = X.xpotrf(limbs, "L", n, expect, n)
    raw, ginfo, _ = KernelContext().mp_potrf(limbs, "L", n, X.pack_array(A), n)
    assert info == ginfo == 6
    got = X.unpack_array(limbs, raw)
    for j in range(5):  # the completed columns agree
        for i in range(j, n):
            assert got[i + j * n] == expect[i + j * n]
