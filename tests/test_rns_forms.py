"""Exact forms of small factors on the GPU: diag_congruence, svec_quadratic, symmetric_bilinear
and gemm_blocks_upper (crates/solver/src/algebra/dense/blas/rns_blas.rs 2990-3194, 4025-4174,
4175-4277, 2656-2923).  Every output is one exact sum of products rounded once, so the GPU result
must be bitwise equal to the oracle's exact restatement (oracle/exact.py).  Inputs come from the
reference's test generator (rns_blas_tests.rs:4-28); the diag_congruence and svec_quadratic
cases are the reference's own (rns_blas_tests.rs:640-642, 742-748)."""
from fractions import Fraction

import pytest

from oracle import exact as X

# (limbs, m, k, spread, seed): rns_blas_tests.rs:742-748 (d drawn with three times the spread)
DIAG_CASES = [(2, 5, 200, 30, 21), (4, 7, 300, 40, 22), (2, 3, 5000, 20, 23), (2, 3, 9000, 20, 24)]
# (limbs, h, kmax, spread, seed): rns_blas_tests.rs:640-642
SVEC_CASES = [(4, 12, 20, 20, 31), (12, 45, 90, 30, 32)]
BILINEAR_CASES = [(4, 10, 16, 20, 41, 30), (2, 1, 3, 5, 42, 4), (8, 24, 9, 40, 43, 12)]
BLOCK_CASES = [(4, 12, [(5, [0, 2, 3, 7, 11]), (7, [1, 2, 3]), (4, [0, 5, 6, 7, 8, 9, 10, 11])], 15, 51),
               (2, 6, [(3, [0, 1, 2, 3, 4, 5]), (0, [1, 2]), (2, [])], 8, 52)]


def _same(got, expect):
    bad = [(i, g, e) for i, (g, e) in enumerate(zip(got, expect)) if not g == e]
    assert not bad, bad[:3]


def test_oracle_diag_congruence_is_the_exact_sum():
    rng = X.Lcg(7)
    n, m, k = 2, 3, 6
    A = X.random_values(n, rng, k * m, 6)
    d = X.random_values(n, rng, k, 18)
    C = X.diag_congruence(n, m, k, A, k, d)
    for j in range(m):
        for i in range(m):
            e = sum(A[r + i * k].fraction() * d[r].fraction() * A[r + j * k].fraction() for r in range(k))
            assert C[i + j * m] == X.from_fraction(n, e)


def test_oracle_bilinear_and_blocks_are_exact_sums():
    rng = X.Lcg(8)
    n, h, cols = 2, 4, 3
    Q = X.random_values(n, rng, h * cols, 5)
    Xp = X.random_values(n, rng, h * (h + 1) // 2, 5)
    got = X.symmetric_bilinear(n, h, Q, Xp, [(0, 2), (1, 1)])
    for (a, b), g in zip([(0, 2), (1, 1)], got):
        e = sum(Q[i + a * h].fraction() * Xp[max(i, j) * (max(i, j) + 1) // 2 + min(i, j)].fraction()
                * Q[j + b * h].fraction() for i in range(h) for j in range(h))
        assert g == X.from_fraction(n, e)
    y = X.random_values(n, rng, 3 * 2, 5)
    d = X.random_values(n, rng, 3, 5)
    out = X.gemm_blocks_upper(n, 4, [(y, d, [1, 3], 3)])
    z = [X.mp_mul(n, d[r], y[r + a * 3]) for a in range(2) for r in range(3)]
    e = sum(z[r + 0 * 3].fraction() * y[r + 1 * 3].fraction() for r in range(3))
    assert out[1 + 3 * 4] == X.from_fraction(n, e)
    assert out[3 + 1 * 4].is_zero()


def test_oracle_sqrt2_is_correctly_rounded():
    for n in (1, 2, 4, 12):
        s = X.sqrt2(n).fraction()
        ulp = Fraction(1, 2 ** (64 * n - 1))
        assert abs(s * s - 2) < 2 * ulp * 2


@pytest.mark.gpu
@pytest.mark.parametrize("n,m,k,spread,seed", DIAG_CASES)
def test_diag_congruence_bitwise(n, m, k, spread, seed):
    from sdpx_b200.solver import KernelContext
    rng = X.Lcg(seed)
    A = X.random_values(n, rng, k * m, spread)
    d = X.random_values(n, rng, k, 3 * spread)
    expect = X.diag_congruence(n, m, k, A, k, d)
    ctx = KernelContext()
    raw, st = ctx.rns_diag_congruence(n, m, k, X.pack_array(A), k, X.pack_array(d))
    assert st == 0
    _same(X.unpack_array(n, raw), expect)
    raw_u, st = ctx.rns_diag_congruence(n, m, k, X.pack_array(A), k, X.pack_array(d), upper_only=True)
    up = X.unpack_array(n, raw_u)
    for j in range(m):
        for i in range(m):
            assert up[i + j * m] == expect[i + j * m] if i <= j else up[i + j * m].is_zero()


@pytest.mark.gpu
@pytest.mark.parametrize("n,h,kmax,spread,seed", SVEC_CASES)
def test_svec_quadratic_bitwise(n, h, kmax, spread, seed):
    from sdpx_b200.solver import KernelContext
    rng = X.Lcg(seed)
    Q = X.random_values(n, rng, h * kmax, spread)
    x = X.random_values(n, rng, h * (h + 1) // 2, spread)
    s2 = X.sqrt2(n)
    ctx = KernelContext()
    for abs_q in (False, True):
        expect = X.svec_quadratic(n, h, kmax, Q, x, s2, abs_q=abs_q)
        raw, st = ctx.rns_svec_quadratic(n, h, kmax, X.pack_array(Q), X.pack_array(x), s2.pack(), abs_q=abs_q)
        assert st == 0
        _same(X.unpack_array(n, raw), expect)


@pytest.mark.gpu
@pytest.mark.parametrize("n,h,cols,spread,seed,npairs", BILINEAR_CASES)
def test_symmetric_bilinear_bitwise(n, h, cols, spread, seed, npairs):
    from sdpx_b200.solver import KernelContext
    rng = X.Lcg(seed)
    Q = X.random_values(n, rng, h * cols, spread)
    Xp = X.random_values(n, rng, h * (h + 1) // 2, spread)
    pairs = [(int(rng.next() * cols), int(rng.next() * cols)) for _ in range(npairs)]
    expect = X.symmetric_bilinear(n, h, Q, Xp, pairs)
    raw, st = KernelContext().rns_symmetric_bilinear(n, h, cols, X.pack_array(Q), X.pack_array(Xp), pairs)
    assert st == 0
    _same(X.unpack_array(n, raw), expect)


@pytest.mark.gpu
@pytest.mark.parametrize("n,m,shape,spread,seed", BLOCK_CASES)
def test_gemm_blocks_upper_bitwise(n, m, shape, spread, seed):
    from sdpx_b200.solver import KernelContext
    rng = X.Lcg(seed)
    blocks = []
    for w, cols in shape:
        y = X.random_values(n, rng, w * len(cols), spread)
        d = X.random_values(n, rng, w, 2 * spread)
        blocks.append((y, d, cols, w))
    expect = X.gemm_blocks_upper(n, m, blocks)
    raw, st = KernelContext().rns_gemm_blocks_upper(
        n, m, [(X.pack_array(y), X.pack_array(d), cols, w) for y, d, cols, w in blocks])
    assert st == 0
    _same(X.unpack_array(n, raw), expect)


@pytest.mark.gpu
def test_exact_forms_reject_bad_input():
    from sdpx_b200 import _lib
    from sdpx_b200.solver import KernelContext
    ctx = KernelContext()
    rng = X.Lcg(3)
    Q = X.pack_array(X.random_values(2, rng, 6, 3))
    Xp = X.pack_array(X.random_values(2, rng, 6, 3))
    with pytest.raises(_lib.SdpxError) as e:
        ctx.rns_symmetric_bilinear(2, 3, 2, Q, Xp, [(0, 2)])  # column 2 of a 2-column basis
    assert e.value.code == 1
    y = X.pack_array(X.random_values(2, rng, 4, 3))
    d = X.pack_array(X.random_values(2, rng, 2, 3))
    with pytest.raises(_lib.SdpxError) as e:
        ctx.rns_gemm_blocks_upper(2, 4, [(y, d, [2, 1], 2)])  # columns not increasing
    assert e.value.code == 1
