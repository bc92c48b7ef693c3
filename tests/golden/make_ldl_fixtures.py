"""Generate the MPFR dense LDL' fixtures from the oracle (oracle/exact.py ldl_rec).

Each case is a symmetric, diagonally dominant n x n MpFloat<limbs> matrix drawn with the
reference's test generator (rns_blas_tests.rs:4-28: LCG values at the working precision with an
exponent spread; the diagonal lifted by n 2^spread so every pivot is positive; `matrix` rebuilds
it from the seed), and the oracle's factorisation of it: D^-1 and the unit lower L as packed
element bytes -- the full lower triangle for n <= 64, its SHA-256 for the larger cases (the
fixtures stay small; the GPU test hashes the same bytes).  n = 160 exceeds the reference's
recursion base (128), so the halving, the row solve and the exact trailing product run; n = 300
also halves inside the row solve (k = 150).  One case applies the pivot rule (eps above some
pivots, which then become delta).

    python tests/golden/make_ldl_fixtures.py
"""
from __future__ import annotations

import hashlib
import sys
import time
from fractions import Fraction
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

# (limbs, n, spread, seed, pivot rule)
CASES = [(2, 24, 3, 31, False), (4, 40, 10, 32, False), (8, 17, 6, 33, False), (4, 160, 4, 34, False),
         (4, 300, 4, 35, False), (4, 40, 4, 36, True)]


def matrix(limbs, n, spread, seed):
    from oracle import exact as X
    rng = X.Lcg(seed)
    A = [None] * (n * n)
    vals = X.random_values(limbs, rng, n * (n + 1) // 2, spread)
    t = 0
    for j in range(n):
        for i in range(j, n):
            v = vals[t]
            t += 1
            if i == j:
                v = X.from_fraction(limbs, abs(v.fraction()) + n * (2 ** spread))
            A[i + j * n] = v
            A[j + i * n] = v
    return A


def pivot_rule(limbs, n, spread):
    """(eps, delta): eps = (n + 1/2) 2^spread lies inside the pivots' range (the diagonal is
    n 2^spread plus a value below 2^spread), delta = n 2^spread / 3 keeps the factor's growth
    modest."""
    from oracle import exact as X
    return (X.from_fraction(limbs, (n + Fraction(1, 2)) * 2 ** spread),
            X.from_fraction(limbs, Fraction(n * 2 ** spread, 3)))


def lower_bytes(X, limbs, n, L):
    """The packed lower triangle (diagonal included) of L, column by column."""
    return b"".join(X.pack_array(L[j + j * n:(j + 1) * n]) for j in range(n))


def make(limbs, n, spread, seed, rule):
    from oracle import exact as X
    A = matrix(limbs, n, spread, seed)
    reg = pivot_rule(limbs, n, spread) if rule else None
    t0 = time.perf_counter()
    dinv = X.ldl_rec(limbs, A, n, 0, n, reg)
    dt = time.perf_counter() - t0
    lower = lower_bytes(X, limbs, n, A)
    out = HERE / f"mpldl_l{limbs}_n{n}_s{seed}.npz"
    np.savez_compressed(out, L=np.frombuffer(lower if n <= 64 else b"", dtype=np.uint8),
                        L_sha256=hashlib.sha256(lower).hexdigest(),
                        dinv=np.frombuffer(X.pack_array(dinv), dtype=np.uint8), limbs=limbs, n=n,
                        spread=spread, seed=seed, rule=rule)
    print(f"limbs {limbs} n {n}: {dt:.1f} s -> {out.name}", flush=True)


if __name__ == "__main__":
    for c in CASES:
        if len(sys.argv) == 1 or f"mpldl_l{c[0]}_n{c[1]}_s{c[3]}" in sys.argv[1:]:
            make(*c)
