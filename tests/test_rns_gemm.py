"""Exact MpFloat products (the RNS BLAS under the reference's MPFR path).

CPU part: the oracle's rounding is checked against mpmath (ties to even at 64N bits).
GPU part: sdpxg_rns_gemm must be bitwise equal to the exact dot product rounded once, on the
reference's own test inputs -- its LCG generator, shapes, precisions and exponent spreads
(crates/solver/src/algebra/dense/blas/rns_blas_tests.rs:4-28, 62-144, 225-229), all four
transposes, and the upper-only variant -- in both residue forms: INT8 tensor cores (primes below
2^15 as two signed-byte digits, tcgen05.mma kind::i8) and FP64 (primes below 2^21).  The
device-pointer entry point gives the same bits as the host one.
"""
from fractions import Fraction

import pytest

from oracle import exact as X


def test_oracle_rounding_matches_mpmath():
    mpmath = pytest.importorskip("mpmath")
    rng = X.Lcg(11)
    for n in (1, 2, 4):
        prec = 64 * n
        for _ in range(200):
            num = Fraction(rng.next() * 2 - 1) * 3 ** 40 + Fraction(1, 7)
            den = Fraction(rng.next() + 0.5) * 5 ** 17
            x = num / den
            mine = X.from_fraction(n, x)
            with mpmath.workprec(prec):  # one correctly rounded division of the exact integers
                ref = mpmath.fdiv(x.numerator, x.denominator, rounding="n")
            sign, man, e2, _ = ref._mpf_  # ref = (-1)^sign * man * 2^e2 exactly
            assert mine.fraction() == (-1) ** sign * Fraction(int(man)) * Fraction(2) ** int(e2)


def test_oracle_exact_dot_ties_to_even():
    n = 1
    one = X.from_fraction(n, Fraction(1))
    tiny = X.from_fraction(n, Fraction(1, 2 ** 64))  # exactly half an ulp of 1 at 64 bits
    # 1 + 2^-64 is a tie between 1 and 1 + 2^-63: ties to even keeps 1
    assert X.exact_dot(n, [(one, one), (tiny, one)]) == one
    three = X.from_fraction(n, Fraction(3, 2 ** 65))  # 1.5 half-ulps: rounds up
    up = X.exact_dot(n, [(one, one), (three, one)])
    assert up.fraction() == 1 + Fraction(1, 2 ** 63)


def _case(n, m, ncols, k, spread, seed):
    rng = X.Lcg(seed)
    out = []
    for ta, tb in (("N", "N"), ("T", "N"), ("N", "T"), ("T", "T")):
        ar, ac = (m, k) if ta == "N" else (k, m)
        br, bc = (k, ncols) if tb == "N" else (ncols, k)
        A = X.random_values(n, rng, ar * ac, spread)
        B = X.random_values(n, rng, br * bc, spread)
        out.append((ta, tb, A, ar, B, br))
    return out


# rns_blas_tests.rs:62-69 (shapes, precisions in limbs, spreads, seeds)
REFERENCE_CASES = [(12, 7, 5, 45, 90, 1), (12, 20, 20, 20, 3, 2), (8, 3, 4, 1, 40, 3),
                   (4, 9, 6, 300, 60, 4), (2, 5, 5, 33, 10, 5), (16, 35, 37, 45, 90, 7)]


FORMS = [0, 1]  # INT8 tensor cores, FP64


@pytest.mark.gpu
@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("n,m,ncols,k,spread,seed", REFERENCE_CASES)
def test_rns_gemm_bitwise_reference_cases(n, m, ncols, k, spread, seed, form):
    from sdpx_b200.solver import KernelContext
    ctx = KernelContext()
    ctx.set_rns_form(form)
    for ta, tb, A, ar, B, br in _case(n, m, ncols, k, spread, seed):
        expect = X.gemm(n, ta, tb, m, ncols, k, A, ar, B, br)
        raw, st = ctx.rns_gemm(n, ta, tb, m, ncols, k, X.pack_array(A), ar, X.pack_array(B), br)
        assert st == 0
        got = X.unpack_array(n, raw)
        bad = [(i, g, e) for i, (g, e) in enumerate(zip(got, expect)) if not g == e]
        assert not bad, (ta, tb, bad[:3])
        # upper-only: the entries i <= j are the same bits
        raw_u, _ = ctx.rns_gemm(n, ta, tb, m, ncols, k, X.pack_array(A), ar, X.pack_array(B), br,
                                upper_only=True)
        up = X.unpack_array(n, raw_u)
        for j in range(ncols):
            for i in range(min(j + 1, m)):
                assert up[i + j * m] == expect[i + j * m]


@pytest.mark.gpu
@pytest.mark.parametrize("form", FORMS)
def test_rns_gemm_long_inner_dimension(form):
    """check::<4>(2, 3, 70_000, 4, 6) (rns_blas_tests.rs:225-229), all four transposes: the INT8
    form splits K into two tensor-core passes (2^16 per pass), the FP64 form reduces every 8192
    terms."""
    from sdpx_b200.solver import KernelContext
    n, m, ncols, k = 4, 2, 3, 70000
    ctx = KernelContext()
    ctx.set_rns_form(form)
    for ta, tb, A, ar, B, br in _case(n, m, ncols, k, 4, 6):
        expect = X.gemm(n, ta, tb, m, ncols, k, A, ar, B, br)
        raw, st = ctx.rns_gemm(n, ta, tb, m, ncols, k, X.pack_array(A), ar, X.pack_array(B), br)
        assert st == 0
        assert all(g == e for g, e in zip(X.unpack_array(n, raw), expect)), (ta, tb)


@pytest.mark.gpu
def test_rns_gemm_device_entry_matches_host_entry():
    """sdpxg_rns_gemm_device on device-resident MpFloat arrays gives the host entry's bits."""
    import numpy as np
    import torch
    from sdpx_b200.solver import KernelContext
    n, m, ncols, k = 4, 35, 37, 45
    (ta, tb, A, ar, B, br), = _case(n, m, ncols, k, 90, 7)[:1]
    ctx = KernelContext()
    host, st = ctx.rns_gemm(n, ta, tb, m, ncols, k, X.pack_array(A), ar, X.pack_array(B), br)
    esz = 8 * n + 8
    dA = torch.from_numpy(np.frombuffer(X.pack_array(A), dtype=np.uint8).copy()).cuda()
    dB = torch.from_numpy(np.frombuffer(X.pack_array(B), dtype=np.uint8).copy()).cuda()
    dC = torch.zeros(m * ncols * esz, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    st2 = ctx.rns_gemm_device(n, ta, tb, m, ncols, k, dA.data_ptr(), ar, dB.data_ptr(), br,
                              dC.data_ptr())
    assert st == st2 == 0
    assert dC.cpu().numpy().tobytes() == host


@pytest.mark.gpu
@pytest.mark.parametrize("form", FORMS)
def test_rns_gemm_cancellation_and_zero(form):
    """Exact cancellation gives zero; a tiny remainder survives the cancellation exactly."""
    from sdpx_b200.solver import KernelContext
    n = 4
    big = X.from_fraction(n, Fraction(3, 7) * 2 ** 200)
    nbig = X.from_fraction(n, -Fraction(3, 7) * 2 ** 200)
    one = X.from_fraction(n, Fraction(1))
    tiny = X.from_fraction(n, Fraction(1, 3) * Fraction(1, 2 ** 300))
    A = [big, nbig, tiny]  # 1 x 3
    B = [one, one, one]  # 3 x 1
    ctx = KernelContext()
    ctx.set_rns_form(form)
    raw, st = ctx.rns_gemm(n, "N", "N", 1, 1, 3, X.pack_array(A), 1, X.pack_array(B), 3)
    got = X.unpack_array(n, raw)[0]
    assert got == tiny
    raw, st = ctx.rns_gemm(n, "N", "N", 1, 1, 2, X.pack_array(A[:2]), 1, X.pack_array(B[:2]), 2)
    assert X.unpack_array(n, raw)[0].is_zero()


# congruence cases: (limbs, m, k, spread, seed, ta); inputs from the reference's generator
CONGRUENCE_CASES = [(4, 5, 7, 4, 11, "N"), (2, 6, 9, 60, 12, "T"), (8, 3, 4, 10, 13, "N"),
                    (4, 12, 20, 30, 14, "T")]


@pytest.mark.gpu
@pytest.mark.parametrize("n,m,k,spread,seed,ta", CONGRUENCE_CASES)
def test_rns_congruence_bitwise(n, m, k, spread, seed, ta):
    """sdpxg_rns_congruence: op(A) X op(A)' with every entry the exact triple sum rounded once
    (rns_blas.rs:3563-3736), against the oracle's exact restatement; upper-only too."""
    from sdpx_b200.solver import KernelContext
    rng = X.Lcg(seed)
    ar, ac = (m, k) if ta == "N" else (k, m)
    A = X.random_values(n, rng, ar * ac, spread)
    Xm = X.random_values(n, rng, k * k, spread)
    expect = X.congruence(n, ta, m, k, A, ar, Xm, k)
    ctx = KernelContext()
    raw, st = ctx.rns_congruence(n, ta, m, k, X.pack_array(A), ar, X.pack_array(Xm), k)
    assert st == 0
    got = X.unpack_array(n, raw)
    bad = [(i, g, e) for i, (g, e) in enumerate(zip(got, expect)) if not g == e]
    assert not bad, bad[:3]
    raw_u, _ = ctx.rns_congruence(n, ta, m, k, X.pack_array(A), ar, X.pack_array(Xm), k, upper_only=True)
    up = X.unpack_array(n, raw_u)
    for j in range(m):
        for i in range(m):
            if i <= j:
                assert up[i + j * m] == expect[i + j * m]
            else:
                assert up[i + j * m].is_zero()


def test_oracle_congruence_matches_products():
    """The oracle's congruence equals the exact rational triple product rounded once."""
    rng = X.Lcg(3)
    n, m, k = 2, 3, 4
    A = X.random_values(n, rng, m * k, 5)
    Xm = X.random_values(n, rng, k * k, 5)
    C = X.congruence(n, "N", m, k, A, m, Xm, k)
    for j in range(m):
        for i in range(m):
            exact = sum(A[i + a * m].fraction() * Xm[a + b * k].fraction() * A[j + b * m].fraction()
                        for a in range(k) for b in range(k))
            assert C[i + j * m] == X.from_fraction(n, exact)
