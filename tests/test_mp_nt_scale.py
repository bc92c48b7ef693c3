"""NT scaling of PSD blocks at MPFR width on the GPU (sdpxg_mp_nt_scale), against the oracle's
restatement of update_scaling (crates/solver/src/solver/cones/psdtrianglecone.rs:311-439;
oracle/exact.py nt_scale).

The right singular vectors come from different methods (one-sided Jacobi in MpFloat on the GPU,
mpmath's SVD in the oracle, Golub-Kahan/dqds in the reference), so V agrees only up to column
signs.  The bars are on what the scaling defines, at working precision 2^-64N:
  * lambda (descending) against the oracle's to 2^-(64N-24) relative;
  * G = R R' against the oracle's to 2^-(64N-24) of max |G| (G does not depend on V's signs);
  * the NT identities of the GPU's own R, Rinv: Rinv R = I, R' Z R = diag(lambda) and
    Rinv S Rinv' = diag(lambda), evaluated in 64N + 64-bit arithmetic, to 2^-(64N-24) relative to
    lambda's scale, including a block whose eigenvalues spread over 2^-100;
  * Lambda^-1/2 = 1 / sqrt(lambda) to 2^-(64N-4);
  * a block with z outside the cone reports status 1 with zero outputs and leaves the others
    intact.
"""
from fractions import Fraction

import numpy as np
import pytest

from oracle import exact as X


def _svec_mp(n, M):
    """svec (upper, column order, off-diagonal times sqrt 2) of an exact symmetric matrix given
    as Fractions, each entry rounded once to 64n bits (the off-diagonal sqrt 2 in 64n + 64-bit
    arithmetic before the rounding)."""
    import mpmath
    k = len(M)
    out = []
    with mpmath.workprec(64 * n + 64):
        r2 = mpmath.sqrt(2)
        for j in range(k):
            for i in range(j + 1):
                v = M[i][j]
                if i == j:
                    out.append(X.from_fraction(n, v))
                else:
                    w = mpmath.mpf(v.numerator) / v.denominator * r2
                    out.append(X.from_fraction(n, X._mpf_fraction(w)))
    return out


def _spd(rng, k, spread_bits=0):
    """L L' for a random lower L whose diagonal spreads over 2^-spread_bits, exact."""
    L = [[Fraction(0)] * k for _ in range(k)]
    for i in range(k):
        L[i][i] = Fraction(1, 2 ** int(spread_bits * i / max(k - 1, 1)))
        for j in range(i):
            L[i][j] = Fraction(float(rng.standard_normal())) / 4 * L[j][j]
    return [[sum(L[i][q] * L[j][q] for q in range(k)) for j in range(k)] for i in range(k)]


def _case(n, orders, seed, spread_bits=0, bad=None):
    rng = np.random.default_rng(seed)
    s, z, mats = [], [], []
    for b, k in enumerate(orders):
        S = _spd(rng, k, spread_bits)
        Z = _spd(rng, k, spread_bits)
        if b == bad:
            Z = [[-v if i == j else v for j, v in enumerate(row)] for i, row in enumerate(Z)]
        sv, zv = _svec_mp(n, S), _svec_mp(n, Z)
        s += sv
        z += zv
        mats.append((sv, zv))
    return s, z, mats


def _mpmat(vals, k):
    import mpmath
    M = mpmath.matrix(k, k)
    for j in range(k):
        for i in range(k):
            f = vals[i + j * k].fraction()
            M[i, j] = mpmath.mpf(f.numerator) / f.denominator
    return M


def _smat(svec_vals, k):
    import mpmath
    M = mpmath.matrix(k, k)
    r = mpmath.sqrt(2)
    for j in range(k):
        for i in range(j + 1):
            f = svec_vals[j * (j + 1) // 2 + i].fraction()
            v = mpmath.mpf(f.numerator) / f.denominator
            M[i, j] = M[j, i] = v if i == j else v / r
    return M


def _check_identities(n, k, sv, zv, lam, R, Rinv):
    import mpmath
    with mpmath.workprec(64 * n + 64):
        Rm, Ri = _mpmat(R, k), _mpmat(Rinv, k)
        S, Z = _smat(sv, k), _smat(zv, k)
        lm = [mpmath.mpf(v.fraction().numerator) / v.fraction().denominator for v in lam]
        D = mpmath.diag(lm)
        tol = mpmath.mpf(2) ** -(64 * n - 24)
        scale = max(abs(v) for v in lm)
        assert mpmath.mnorm(Ri * Rm - mpmath.eye(k), 1) <= tol * k
        assert mpmath.mnorm(Rm.T * Z * Rm - D, 1) <= tol * scale * k
        assert mpmath.mnorm(Ri * S * Ri.T - D, 1) <= tol * scale * k


def test_oracle_nt_scale_identities():
    n = 4
    s, z, mats = _case(n, [1, 3, 6], seed=1, spread_bits=40)
    for k, (sv, zv) in zip([1, 3, 6], mats):
        lam, lis, R, Rinv, G = X.nt_scale(n, k, sv, zv)
        _check_identities(n, k, sv, zv, lam, R, Rinv)


@pytest.mark.gpu
@pytest.mark.parametrize("n,orders,seed,spread", [(2, [1, 2, 3, 7, 20], 3, 0), (4, [5, 12, 60], 4, 0),
                                                  (4, [2, 9, 16], 5, 100), (8, [4, 11], 6, 60)])
def test_mp_nt_scale_matches_oracle(n, orders, seed, spread):
    from sdpx_b200.solver import KernelContext
    s, z, mats = _case(n, orders, seed, spread)
    lam_b, lis_b, R_b, Ri_b, G_b, bst, st = KernelContext().mp_nt_scale(n, orders, X.pack_array(s),
                                                                          X.pack_array(z))
    assert st == 0 and bst == [0] * len(orders)
    lam_all, lis_all = X.unpack_array(n, lam_b), X.unpack_array(n, lis_b)
    R_all, Ri_all, G_all = X.unpack_array(n, R_b), X.unpack_array(n, Ri_b), X.unpack_array(n, G_b)
    lo = sq = 0
    tol = Fraction(1, 2 ** (64 * n - 24))
    for k, (sv, zv) in zip(orders, mats):
        lam, lis = lam_all[lo:lo + k], lis_all[lo:lo + k]
        R, Rinv, G = R_all[sq:sq + k * k], Ri_all[sq:sq + k * k], G_all[sq:sq + k * k]
        olam, _, _, _, oG = X.nt_scale(n, k, sv, zv)
        for a, b in zip(lam, olam):
            assert abs(a.fraction() - b.fraction()) <= tol * abs(b.fraction())
        for a, b in zip(lam, lis):
            assert abs(b.fraction() ** 2 * a.fraction() - 1) <= Fraction(1, 2 ** (64 * n - 4))
        gmax = max(abs(v.fraction()) for v in oG)
        for j in range(k):
            for i in range(k):
                a, b = G[i + j * k], oG[i + j * k]
                if i > j:
                    assert a.is_zero()
                else:
                    assert abs(a.fraction() - b.fraction()) <= tol * gmax
        _check_identities(n, k, sv, zv, lam, R, Rinv)
        lo += k
        sq += k * k


@pytest.mark.gpu
def test_mp_nt_scale_reports_a_block_outside_the_cone():
    from sdpx_b200.solver import KernelContext
    n, orders = 4, [3, 5, 4]
    s, z, mats = _case(n, orders, 7, 0, bad=1)
    lam_b, _, _, _, _, bst, st = KernelContext().mp_nt_scale(n, orders, X.pack_array(s), X.pack_array(z))
    assert bst == [0, 1, 0] and st == 0
    lam = X.unpack_array(n, lam_b)
    assert all(v.is_zero() for v in lam[3:8])
    olam = X.nt_scale(n, 4, *mats[2])[0]
    tol = Fraction(1, 2 ** (64 * n - 24))
    for a, b in zip(lam[8:12], olam):
        assert abs(a.fraction() - b.fraction()) <= tol * abs(b.fraction())
