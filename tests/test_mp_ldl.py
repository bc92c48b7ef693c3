"""The reference's dense MPFR LDL' on the GPU (sdpxg_mp_ldl), bitwise against the oracle.

The oracle (oracle/exact.py ldl_rec / ldl_dots / solve_unit_lower_t) restates
crates/solver/src/solver/kkt/ldl/arrow.rs:156-470 with every operation exact and rounded once to
64N bits (ties to even); its outputs on the reference's own test generator are committed as
fixtures (tests/golden/make_ldl_fixtures.py).  The GPU factor must give the same bits: the unit
lower L and D^-1, on single leaves (n <= 128, the exact-dot kernel), one halving (n = 160: the
row solve, the scaling and the exact trailing product on the INT8 tensor cores) and a halving
whose row solve halves again (n = 300), at 128, 256 and 512 bits, with and without the pivot
rule.
"""
import hashlib
import sys
from pathlib import Path

import numpy as np
import pytest

from oracle import exact as X

GOLDEN = Path(__file__).resolve().parent / "golden"
sys.path.insert(0, str(GOLDEN))
import make_ldl_fixtures as F  # noqa: E402  (rebuilds each case's matrix from its seed)

CASES = sorted(p.name for p in GOLDEN.glob("mpldl_*.npz"))


def test_ldl_fixtures_present_and_oracle_reproduces_small_case():
    assert len(CASES) >= 6
    fx = np.load(GOLDEN / "mpldl_l2_n24_s31.npz")
    n, limbs = int(fx["n"]), int(fx["limbs"])
    A0 = F.matrix(limbs, n, int(fx["spread"]), int(fx["seed"]))
    A = list(A0)
    dinv = X.ldl_rec(limbs, A, n, 0, n)
    lower = F.lower_bytes(X, limbs, n, A)
    assert lower == fx["L"].tobytes()
    assert hashlib.sha256(lower).hexdigest() == str(fx["L_sha256"])
    assert X.pack_array(dinv) == fx["dinv"].tobytes()
    # L D L' reproduces the matrix to the working precision
    Lf = np.array([[float(A[i + j * n].fraction()) if i >= j else 0.0 for j in range(n)] for i in range(n)])
    D = np.diag([1.0 / float(d.fraction()) for d in dinv])
    Af = np.array([[float(A0[i + j * n].fraction()) for j in range(n)] for i in range(n)])
    assert np.max(np.abs(Lf @ D @ Lf.T - Af)) <= 1e-12 * np.max(np.abs(Af))


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_mp_ldl_bitwise(name):
    from sdpx_b200.solver import KernelContext
    fx = np.load(GOLDEN / name)
    n, limbs, spread = int(fx["n"]), int(fx["limbs"]), int(fx["spread"])
    A = F.matrix(limbs, n, spread, int(fx["seed"]))
    reg = X.pack_array(list(F.pivot_rule(limbs, n, spread))) if bool(fx["rule"]) else None
    L, dinv, st = KernelContext().mp_ldl(limbs, n, X.pack_array(A), n, reg)
    assert st == 0
    got = X.unpack_array(limbs, L)
    # zeros compare by value (the sign of a zero is not part of the contract)
    lower = F.lower_bytes(X, limbs, n, [X.Mp(limbs) if v.is_zero() else v for v in got])
    if fx["L"].size:
        exp = X.unpack_array(limbs, fx["L"].tobytes())
        gl = X.unpack_array(limbs, lower)
        bad = [k for k, (g, e) in enumerate(zip(gl, exp)) if not g == e]
        assert not bad, bad[:5]
    assert hashlib.sha256(lower).hexdigest() == str(fx["L_sha256"])
    assert all(g == e for g, e in zip(X.unpack_array(limbs, dinv), X.unpack_array(limbs, fx["dinv"].tobytes())))
