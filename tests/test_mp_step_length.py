"""Step-length bounds of PSD blocks at MPFR width on the GPU (sdpxg_mp_step_length) against the
oracle's restatement (oracle/exact.py step_component; psdtrianglecone.rs:1041-1072, 1180-1390).

Bars: the path taken (a priori binary64 bound, exact Cholesky certificate, full-precision
eigensolver) equals the oracle's; on the binary64 paths alpha is bitwise equal (the same binary64
eigenvalue, the same correctly rounded reciprocal); on the eigensolver path alpha agrees to
2^-(64N-24) relative (a Jacobi eigensolver on the GPU, mpmath's in the oracle).  Directions are
given with identity scaling (so their spectra, and with them the paths, are chosen) and with the
NT scaling of random interior points, on both the primal (Rinv) and the dual (R) side."""
from fractions import Fraction

import numpy as np
import pytest

from oracle import exact as X


def _svec_f64(M):
    k = M.shape[0]
    return [M[i, j] if i == j else M[i, j] * np.sqrt(2.0) for j in range(k) for i in range(j + 1)]


def _direction(rng, k, spectrum):
    Q, _ = np.linalg.qr(rng.standard_normal((k, k)))
    return Q @ np.diag(spectrum) @ Q.T


def _identity_blocks(n):
    """(order, direction svec, R, lisqrt) with identity scaling; spectra chosen for each path."""
    rng = np.random.default_rng(17)
    specs = [
        np.concatenate([[-1.0], rng.uniform(-0.5, 2.0, 7)]),          # a priori bound
        rng.uniform(0.1, 1.0, 6),                                     # no negative eigenvalue
        np.concatenate([[-1e-2], rng.uniform(0.5, 1.5, 39)]),         # certificate
        np.array([0.3, -0.7, 0.2]),                                   # order 3: eigensolver
        np.array([-2.5]),                                             # order 1
    ]
    out = []
    one = X.mp_one(n)
    for sp in specs:
        k = len(sp)
        D = _direction(rng, k, sp)
        d = [X.mp_from_float(n, v) for v in _svec_f64(D)]
        R = [one if i == j else X.Mp(n) for j in range(k) for i in range(k)]
        out.append((k, d, R, [one] * k))
    return out


def _nt_blocks(n, primal):
    rng = np.random.default_rng(23 + primal)
    out = []
    for k in (5, 12):
        A = rng.standard_normal((k, k))
        S = A @ A.T / k + 0.3 * np.eye(k)
        B = rng.standard_normal((k, k))
        Z = B @ B.T / k + 0.3 * np.eye(k)
        s = [X.mp_from_float(n, v) for v in _svec_f64(S)]
        z = [X.mp_from_float(n, v) for v in _svec_f64(Z)]
        lam, lis, R, Rinv, _ = X.nt_scale(n, k, s, z)
        D = _direction(rng, k, rng.uniform(-1.0, 1.0, k))
        d = [X.mp_from_float(n, v) for v in _svec_f64(D)]
        out.append((k, d, Rinv if primal else R, lis))
    return out


def _oracle(n, blocks, primal, amax):
    return [X.step_component(n, k, d, R, lis, primal, amax) for k, d, R, lis in blocks]


def test_oracle_step_paths_cover_the_certificate():
    n = 4
    res = _oracle(n, _identity_blocks(n), False, X.mp_from_float(n, 1e12))
    assert [p for _, p in res] == [0, 0, 1, 2, 2]
    # the certified bound is min(-1/gamma, alpha_max) with gamma the binary64 eigenvalue
    assert abs(float(res[2][0].fraction()) - 100.0) < 1e-6
    # order 1: alpha = -1/d exactly rounded
    assert res[4][0] == X.mp_recip(n, X.mp_from_float(n, 2.5))


def test_oracle_min_eigenvalue_f64_matches_lapack():
    rng = np.random.default_rng(3)
    for k in (4, 9, 30):
        A = rng.standard_normal((k, k))
        A = A + A.T
        g = X.min_eigenvalue_f64(list(A.T.ravel()), k)
        assert abs(g - np.linalg.eigvalsh(A)[0]) <= 1e-12 * np.max(np.abs(A)) * k


def _run(n, blocks, primal, amax):
    from sdpx_b200.solver import KernelContext
    orders = [k for k, _, _, _ in blocks]
    d = X.pack_array([v for _, dd, _, _ in blocks for v in dd])
    R = X.pack_array([v for _, _, RR, _ in blocks for v in RR])
    lis = X.pack_array([v for _, _, _, ll in blocks for v in ll])
    raw, path, st = KernelContext().mp_step_length(n, orders, primal, d, R, lis, amax.pack())
    assert st == 0
    return X.unpack_array(n, raw), path


@pytest.mark.gpu
@pytest.mark.parametrize("n", [2, 4])
def test_mp_step_length_identity_scaling(n):
    amax = X.mp_from_float(n, 1e12)
    blocks = _identity_blocks(n)
    alpha, path = _run(n, blocks, False, amax)
    expect = _oracle(n, blocks, False, amax)
    assert path == [p for _, p in expect]
    for a, (e, p) in zip(alpha, expect):
        if p < 2:
            assert a == e
        else:
            assert abs(a.fraction() - e.fraction()) <= Fraction(1, 2 ** (64 * n - 24)) * abs(e.fraction())


@pytest.mark.gpu
@pytest.mark.parametrize("primal", [False, True])
def test_mp_step_length_nt_scaled(primal):
    n = 4
    amax = X.mp_one(n)
    blocks = _nt_blocks(n, primal)
    alpha, path = _run(n, blocks, primal, amax)
    expect = _oracle(n, blocks, primal, amax)
    assert path == [p for _, p in expect]
    for a, (e, p) in zip(alpha, expect):
        if p < 2:
            assert a == e
        else:
            assert abs(a.fraction() - e.fraction()) <= Fraction(1, 2 ** (64 * n - 24)) * abs(e.fraction())
