"""Exact-rounding restatement of the MPFR contract used by the RNS BLAS -- TEST ORACLE.

Test infrastructure only (see ``oracle/__init__``).  Restates, in Python integers:

* ``MpFloat<N>`` (crates/arithmetic/src/lib.rs:333-349): N x 64-bit mantissa limbs, least
  significant first, an i32 MPFR kind whose sign is the value's sign (2 = zero, 3 = regular)
  and an i32 exponent; a regular value is M * 2^(exponent - 64N) with 2^(64N-1) <= M < 2^(64N);
* ``from_scaled_integer`` (crates/arithmetic/src/exactdot.rs:1316-1392): round an exact integer
  times a power of two to 64N bits, ties to even;
* ``dot_fma`` (crates/arithmetic/src/lib.rs:535-545, exactdot.rs:53-70): the exact dot product
  rounded once -- the value every RNS product must reproduce bitwise
  (crates/solver/src/algebra/dense/blas/rns_blas_tests.rs:30-144);
* the reference's RNS test-input generator (rns_blas_tests.rs:4-28): a 64-bit LCG, values
  (2u - 1) / (u + 1/2) rounded at the working precision, 5% zeros, and a power-of-two spread.

Correct rounding is a definition, so this oracle is pinned by it; ``tests/test_oracle_pins.py``
cross-checks the rounding against mpmath.
"""
from __future__ import annotations

import math
import struct
from fractions import Fraction
from typing import List, Sequence, Tuple

ZERO_KIND = 2
REGULAR_KIND = 3
MASK64 = (1 << 64) - 1


class Mp:
    """A finite MpFloat<N> value: (negative, mantissa M, exponent e) or zero."""

    __slots__ = ("n", "neg", "mant", "exp")

    def __init__(self, n: int, neg: bool = False, mant: int = 0, exp: int = 0):
        self.n, self.neg, self.mant, self.exp = n, neg, mant, exp

    @property
    def p(self) -> int:
        return 64 * self.n

    def is_zero(self) -> bool:
        return self.mant == 0

    def fraction(self) -> Fraction:
        if self.mant == 0:
            return Fraction(0)
        v = Fraction(self.mant) * Fraction(2) ** (self.exp - self.p)
        return -v if self.neg else v

    def pack(self) -> bytes:
        limbs = [(self.mant >> (64 * q)) & MASK64 for q in range(self.n)]
        if self.mant == 0:
            return struct.pack(f"<{self.n}Qii", *([0] * self.n), ZERO_KIND, 0)
        kind = -REGULAR_KIND if self.neg else REGULAR_KIND
        return struct.pack(f"<{self.n}Qii", *limbs, kind, self.exp)

    @staticmethod
    def unpack(n: int, raw: bytes) -> "Mp":
        vals = struct.unpack(f"<{n}Qii", raw)
        limbs, kind, exp = vals[:n], vals[n], vals[n + 1]
        if abs(kind) == ZERO_KIND:
            return Mp(n)
        if abs(kind) != REGULAR_KIND:
            raise ValueError(f"non-finite kind {kind}")
        mant = sum(int(l) << (64 * q) for q, l in enumerate(limbs))
        return Mp(n, kind < 0, mant, exp)

    def __eq__(self, other) -> bool:
        if self.is_zero() or other.is_zero():
            return self.is_zero() and other.is_zero()
        return (self.neg, self.mant, self.exp) == (other.neg, other.mant, other.exp)

    def __repr__(self) -> str:
        return f"Mp({'-' if self.neg else '+'}{self.mant:#x}*2^({self.exp}-{self.p}))"


def from_scaled_integer(n: int, negative: bool, mag: int, scale: int) -> Mp:
    """Round mag * 2^scale to 64n bits, ties to even (exactdot.rs:1316-1392)."""
    if mag == 0:
        return Mp(n)
    p = 64 * n
    bits = mag.bit_length()
    shift = bits - p
    if shift > 0:
        top = mag >> shift
        round_bit = (mag >> (shift - 1)) & 1
        sticky = (mag & ((1 << (shift - 1)) - 1)) != 0
        if round_bit and (sticky or (top & 1)):
            top += 1
            if top >> p:
                top >>= 1
                shift += 1
        mant = top
    else:
        mant = mag << (-shift)
    return Mp(n, negative, mant, scale + shift + p)


def from_fraction(n: int, x: Fraction) -> Mp:
    """Correctly rounded (ties to even) 64n-bit value of a rational."""
    if x == 0:
        return Mp(n)
    neg = x < 0
    x = abs(x)
    p = 64 * n
    num, den = x.numerator, x.denominator
    # choose s with 2^(p+2) <= num * 2^s / den so the quotient carries guard bits
    s = p + 2 - (num.bit_length() - den.bit_length()) + 1
    if s >= 0:
        q, r = divmod(num << s, den)
    else:
        q, r = divmod(num, den << (-s))
    # q * 2^-s + r / den * 2^-s; fold the remainder into a sticky bit
    mag = (q << 1) | (1 if r else 0)
    return from_scaled_integer(n, neg, mag, -s - 1)


def exact_dot(n: int, pairs: Sequence[Tuple[Mp, Mp]]) -> Mp:
    """sum a*b computed exactly and rounded once (the dot_fma contract)."""
    terms = [(a, b) for a, b in pairs if not a.is_zero() and not b.is_zero()]
    if not terms:
        return Mp(n)
    low = min((a.exp - a.p) + (b.exp - b.p) for a, b in terms)
    total = 0
    for a, b in terms:
        v = (a.mant * b.mant) << ((a.exp - a.p) + (b.exp - b.p) - low)
        total += -v if (a.neg != b.neg) else v
    return from_scaled_integer(n, total < 0, abs(total), low)


def gemm(n: int, ta: str, tb: str, m: int, ncols: int, k: int, A: List[Mp], lda: int,
         B: List[Mp], ldb: int) -> List[Mp]:
    """C = op(A) op(B) with every entry an exact dot rounded once (rns_blas_tests.rs:30-59)."""
    def at(i, q):
        return A[i + q * lda] if ta == "N" else A[q + i * lda]

    def bt(q, j):
        return B[q + j * ldb] if tb == "N" else B[j + q * ldb]

    return [exact_dot(n, [(at(i, q), bt(q, j)) for q in range(k)])
            for j in range(ncols) for i in range(m)]


class Lcg:
    """The reference's test generator (rns_blas_tests.rs:4-13)."""

    def __init__(self, seed: int):
        self.s = seed & MASK64

    def next(self) -> float:
        self.s = (self.s * 6364136223846793005 + 1442695040888963407) & MASK64
        return (self.s >> 11) / float(1 << 53)


def random_values(n: int, rng: Lcg, length: int, spread: int) -> List[Mp]:
    """rns_blas_tests.rs:15-28: 5% zeros, (2u-1)/(u+1/2) at 64n bits, times 2^shift."""
    out = []
    for _ in range(length):
        if rng.next() < 0.05:
            out.append(Mp(n))
            continue
        num = Fraction(rng.next() * 2.0 - 1.0)
        den = Fraction(rng.next() + 0.5)
        shift = int(rng.next() * (2 * spread + 1)) - spread
        q = from_fraction(n, num / den)
        if not q.is_zero():
            q.exp += shift
        out.append(q)
    return out


def pack_array(vals: Sequence[Mp]) -> bytes:
    return b"".join(v.pack() for v in vals)


def unpack_array(n: int, raw: bytes) -> List[Mp]:
    size = 8 * n + 8
    return [Mp.unpack(n, raw[i * size:(i + 1) * size]) for i in range(len(raw) // size)]


def exact_sum_of_products(n: int, factors: Sequence[Sequence[Mp]]) -> Mp:
    """sum over terms of the product of each term's factors, exact, rounded once."""
    terms = [t for t in factors if all(not f.is_zero() for f in t)]
    if not terms:
        return Mp(n)

    def scale(t):
        return sum(f.exp - f.p for f in t)
    low = min(scale(t) for t in terms)
    total = 0
    for t in terms:
        v = 1
        neg = False
        for f in t:
            v *= f.mant
            neg ^= f.neg
        v <<= scale(t) - low
        total += -v if neg else v
    return from_scaled_integer(n, total < 0, abs(total), low)


def congruence(n: int, ta: str, m: int, k: int, A: List[Mp], lda: int, X: List[Mp], ldx: int,
               upper_only: bool = False) -> List[Mp]:
    """C = op(A) X op(A)' with every entry the exact triple sum rounded once
    (crates/solver/src/algebra/dense/blas/rns_blas.rs:3563-3736 congruence; op(A) is m x k, X is
    k x k, C column-major m x m; upper_only leaves zeros below the diagonal)."""
    def at(i, q):
        return A[i + q * lda] if ta == "N" else A[q + i * lda]
    out = []
    for j in range(m):
        for i in range(m):
            if upper_only and i > j:
                out.append(Mp(n))
                continue
            out.append(exact_sum_of_products(
                n, [(at(i, a), X[a + b * ldx], at(j, b)) for a in range(k) for b in range(k)]))
    return out


# ------------------------------------------------------------------------------------------
# MpFloat arithmetic (each operation exact, then rounded once to 64n bits, ties to even: the
# MPFR contract of crates/arithmetic/src/lib.rs) and the reference's dense MPFR LDL'
# (crates/solver/src/solver/kkt/ldl/arrow.rs:156-242 ldl_dots, 255-420 ldl_rec,
# 430-470 solve_unit_lower_t) for a dense matrix (row envelope all zero, no cut, sign +1).
# ------------------------------------------------------------------------------------------
REC_BASE = 128  # arrow.rs:63


def mp_sub(n: int, a: Mp, b: Mp) -> Mp:
    return from_fraction(n, a.fraction() - b.fraction())


def mp_mul(n: int, a: Mp, b: Mp) -> Mp:
    return from_fraction(n, a.fraction() * b.fraction())


def mp_recip(n: int, d: Mp) -> Mp:
    return from_fraction(n, 1 / d.fraction())


def mp_from_float(n: int, x: float) -> Mp:
    return from_fraction(n, Fraction(x))


def mp_one(n: int) -> Mp:
    return Mp(n, False, 1 << (64 * n - 1), 1)


def _pivot(d: Mp, reg):
    """DenseLeaf::pivot (arrow.rs:618-632) with sign +1: below eps becomes delta; zero fails."""
    if reg is not None:
        eps, delta = reg
        if d.fraction() < eps.fraction():
            d = delta
    if d.is_zero():
        raise ArithmeticError("zero_pivot")
    return d


def ldl_dots(n: int, A: List[Mp], lda: int, off: int, size: int, reg=None):
    """arrow.rs:156-242 on the diagonal block at (off, off) of A (column-major, lower triangle
    read and overwritten with the unit lower L); returns the block's D^-1.  Every dot is exact
    and rounded once; differences, products and the reciprocal are rounded once each."""
    def at(i, j):
        return A[off + i + (off + j) * lda]
    r = [[None] * size for _ in range(size)]  # r[i][j] = L(i, j), j < i
    w = [[None] * size for _ in range(size)]  # w[i][j] = L(i, j) d_j
    dinv = [None] * size
    for j in range(size):
        rj = [(r[j][c], w[j][c]) for c in range(j)]
        dj = mp_sub(n, at(j, j), exact_dot(n, rj))
        if dj.is_zero() and rj:  # the exact difference rounded once (arrow.rs:190-197)
            dj = from_fraction(n, at(j, j).fraction() - sum(x.fraction() * y.fraction() for x, y in rj))
        dj = _pivot(dj, reg)
        dinv[j] = mp_recip(n, dj)
        for i in range(j + 1, size):
            dot = exact_dot(n, [(r[i][c], w[j][c]) for c in range(j)])
            v = mp_mul(n, mp_sub(n, at(i, j), dot), dinv[j])
            r[i][j] = v
            w[i][j] = mp_mul(n, v, dj)
    for j in range(size):
        A[off + j + (off + j) * lda] = mp_one(n)
        for i in range(j + 1, size):
            A[off + i + (off + j) * lda] = r[i][j]
    return dinv


def solve_unit_lower_t(n: int, m: int, k: int, L: List[Mp], ldl: int, loff: int, B: List[Mp], ldb: int,
                       boff_r: int, boff_c: int):
    """X L' = B (arrow.rs:430-470) for B m x k at (boff_r, boff_c) of B, L unit lower k x k at
    (loff, loff) of L; X overwrites B."""
    def lt(i, j):
        return L[loff + i + (loff + j) * ldl]

    def bt(i, j):
        return B[boff_r + i + (boff_c + j) * ldb]
    if k <= REC_BASE:
        for i in range(m):
            x = [bt(i, j) for j in range(k)]
            for j in range(k):
                x[j] = mp_sub(n, x[j], exact_dot(n, [(x[c], lt(j, c)) for c in range(j)]))
            for j in range(k):
                B[boff_r + i + (boff_c + j) * ldb] = x[j]
        return
    k1, k2 = k // 2, k - k // 2
    solve_unit_lower_t(n, m, k1, L, ldl, loff, B, ldb, boff_r, boff_c)
    # B2 -= B1 L21' with L21 = L(k1:, :k1), each entry exact and rounded once, then subtracted
    for j in range(k2):
        for i in range(m):
            p = exact_dot(n, [(bt(i, c), lt(k1 + j, c)) for c in range(k1)])
            B[boff_r + i + (boff_c + k1 + j) * ldb] = mp_sub(n, bt(i, k1 + j), p)
    solve_unit_lower_t(n, m, k2, L, ldl, loff + k1, B, ldb, boff_r, boff_c + k1)


def ldl_rec(n: int, A: List[Mp], lda: int, off: int, size: int, reg=None) -> List[Mp]:
    """arrow.rs:255-420 for a dense block (no envelope cut): halves, W21 = A21 L11^-T,
    L21 = W21 D1^-1, then A22(b, a) -= (W21 L21')(a, b) for b >= a (one exact product per
    entry, rounded once, then subtracted), recursion; blocks up to REC_BASE take ldl_dots.
    Returns D^-1."""
    if size <= REC_BASE:
        return ldl_dots(n, A, lda, off, size, reg)
    n1, n2 = size // 2, size - size // 2
    d1 = ldl_rec(n, A, lda, off, n1, reg)
    solve_unit_lower_t(n, n2, n1, A, lda, off, A, lda, off + n1, off)
    W = [[A[off + n1 + i + (off + j) * lda] for j in range(n1)] for i in range(n2)]
    for j in range(n1):
        for i in range(n2):
            A[off + n1 + i + (off + j) * lda] = mp_mul(n, W[i][j], d1[j])
    for a in range(n2):
        for b in range(a, n2):
            p = exact_dot(n, [(W[a][c], A[off + n1 + b + (off + c) * lda]) for c in range(n1)])
            idx = off + n1 + b + (off + n1 + a) * lda
            A[idx] = mp_sub(n, A[idx], p)
    d2 = ldl_rec(n, A, lda, off + n1, n2, reg)
    return d1 + d2


def mp_div(n: int, a: Mp, b: Mp) -> Mp:
    return from_fraction(n, a.fraction() / b.fraction())


def mp_sqrt(n: int, a: Mp) -> Mp:
    """Correctly rounded square root (ties to even) of a >= 0: the integer square root of the
    scaled mantissa with the remainder as a sticky bit."""
    if a.is_zero():
        return Mp(n)
    from math import isqrt
    s = a.exp - a.p  # a = mant 2^s
    e = 64 * n + 4
    if (s - e) % 2:
        e += 1
    X = a.mant << e
    y = isqrt(X)
    sticky = 1 if y * y != X else 0
    return from_scaled_integer(n, False, (y << 1) | sticky, (s - e) // 2 - 1)


def xpotrf(n: int, uplo: str, size: int, A: List[Mp], lda: int) -> int:
    """XpotrfScalar::xpotrf for MpFloat (algebra/dense/blas/mpfr.rs:726-789), in place; returns
    info (0, or j + 1 at the first non-positive pivot)."""
    lower = uplo == "L"

    def at(i, k):
        return i + k * lda if lower else k + i * lda
    for j in range(size):
        d = mp_sub(n, A[j + j * lda], exact_dot(n, [(A[at(j, k)], A[at(j, k)]) for k in range(j)]))
        if d.is_zero() or d.neg:
            A[j + j * lda] = d
            return j + 1
        d = mp_sqrt(n, d)
        A[j + j * lda] = d
        for i in range(j + 1, size):
            solved = exact_dot(n, [(A[at(i, k)], A[at(j, k)]) for k in range(j)])
            A[at(i, j)] = mp_div(n, mp_sub(n, A[at(i, j)], solved), d)
    return 0


# ------------------------------------------------------------------------------------------
# Exact forms of small factors (crates/solver/src/algebra/dense/blas/rns_blas.rs): every output
# is one exact sum of products, rounded once to 64n bits, ties to even.
# ------------------------------------------------------------------------------------------
def mp_abs(a: Mp) -> Mp:
    return Mp(a.n, False, a.mant, a.exp) if not a.is_zero() else Mp(a.n)


def sqrt2(n: int) -> Mp:
    """The working-precision sqrt 2 (correctly rounded; FloatConst::SQRT_2 of MpFloat<n>)."""
    return mp_sqrt(n, mp_from_float(n, 2.0))


def diag_congruence(n: int, m: int, k: int, A: List[Mp], lda: int, d: List[Mp],
                    upper_only: bool = False) -> List[Mp]:
    """C = A' diag(d) A for A k x m column-major (rns_blas.rs:2990-3194 diag_congruence): entry
    (i, j) is sum_r A(r, i) d(r) A(r, j), exact, rounded once; zeros below the diagonal when
    upper_only."""
    out = []
    for j in range(m):
        for i in range(m):
            if upper_only and i > j:
                out.append(Mp(n))
                continue
            out.append(exact_sum_of_products(
                n, [(A[r + i * lda], d[r], A[r + j * lda]) for r in range(k)]))
    return out


def svec_quadratic(n: int, h: int, kmax: int, Q: List[Mp], x: List[Mp], s2: Mp,
                   abs_q: bool = False) -> List[Mp]:
    """v[k] = sum_{i <= j} c_ij x_t q_ik q_jk, t = tri(j) + i, c_ii = 1, c_ij = s2 (the
    working-precision sqrt 2), each exact and rounded once (rns_blas.rs:4025-4174)."""
    q = [mp_abs(v) for v in Q] if abs_q else Q
    out = []
    for k in range(kmax):
        terms = []
        for j in range(h):
            for i in range(j + 1):
                t = j * (j + 1) // 2 + i
                a, b = q[i + k * h], q[j + k * h]
                terms.append((x[t], a, b) if i == j else (s2, x[t], a, b))
        out.append(exact_sum_of_products(n, terms))
    return out


def symmetric_bilinear(n: int, h: int, Q: List[Mp], X: List[Mp],
                       pairs: Sequence[Tuple[int, int]]) -> List[Mp]:
    """q_a' X q_b for each pair, X symmetric packed upper without svec factors
    (rns_blas.rs:4175-4277 symmetric_bilinear), exact, rounded once."""
    def xe(i, j):
        lo, hi = min(i, j), max(i, j)
        return X[hi * (hi + 1) // 2 + lo]
    return [exact_sum_of_products(n, [(Q[i + a * h], xe(i, j), Q[j + b * h])
                                      for i in range(h) for j in range(h)])
            for a, b in pairs]


def gemm_blocks_upper(n: int, m: int, blocks) -> List[Mp]:
    """Upper triangle of sum_b Z_b' Y_b, Z_b = diag(d_b) Y_b rounded entrywise, the sum over all
    blocks and rows exact and rounded once (rns_blas.rs:2656-2923 gemm_blocks_upper); blocks are
    (y, d, columns, w) with y w x len(columns) column-major.  Zeros below the diagonal."""
    terms = {}
    for y, d, cols, w in blocks:
        for a, ca in enumerate(cols):
            for b, cb in enumerate(cols):
                if ca > cb:
                    continue
                lst = terms.setdefault((ca, cb), [])
                for r in range(w):
                    lst.append((mp_mul(n, d[r], y[r + a * w]), y[r + b * w]))
    return [exact_dot(n, terms.get((i, j), [])) if i <= j else Mp(n)
            for j in range(m) for i in range(m)]


# ------------------------------------------------------------------------------------------
# NT scaling of one PSD block at MPFR width (crates/solver/src/solver/cones/
# psdtrianglecone.rs:311-439 update_scaling, svec_to_mat algebra/dense/matrix_math.rs:156-180):
# exact-dot Cholesky of both sides, M = L2' L1 with every entry an exact dot rounded once, its
# right singular vectors (here from mpmath's SVD at twice the width, standing in for the
# reference's MPFR right SVD), then lambda, Lambda^-1/2, R = L1 V Lambda^-1/2,
# Rinv = Lambda^1/2 (L1^-T V)' and G = R R' (upper) with MpFloat operations rounded once.
# ------------------------------------------------------------------------------------------
def _mpf_fraction(x) -> Fraction:
    sign, man, exp, _ = x._mpf_
    v = Fraction(int(man)) * (Fraction(2) ** int(exp))
    return -v if sign else v


def frac_1_sqrt2(n: int) -> Mp:
    return mp_sqrt(n, from_fraction(n, Fraction(1, 2)))


def nt_scale(n: int, order: int, s: List[Mp], z: List[Mp]):
    """Returns (lam, lisqrt, R, Rinv, G) as lists (matrices column-major order x order), or
    None when s or z is not interior (a Cholesky fails)."""
    import mpmath
    k = order
    f = frac_1_sqrt2(n)
    S = [Mp(n)] * (k * k)
    Z = [Mp(n)] * (k * k)
    for j in range(k):
        for i in range(j, k):
            t = i * (i + 1) // 2 + j
            S[i + j * k] = s[t] if i == j else mp_mul(n, s[t], f)
            Z[i + j * k] = z[t] if i == j else mp_mul(n, z[t], f)
    if xpotrf(n, "L", k, S, k) or xpotrf(n, "L", k, Z, k):
        return None
    L1, L2 = S, Z
    M = [exact_dot(n, [(L2[q + i * k], L1[q + j * k]) for q in range(max(i, j), k)])
         for j in range(k) for i in range(k)]
    with mpmath.workprec(128 * n + 64):  # twice the working width: small values keep their digits
        Mm = mpmath.matrix(k, k)
        for j in range(k):
            for i in range(k):
                Mm[i, j] = mpmath.mpf(M[i + j * k].fraction().numerator) / M[i + j * k].fraction().denominator
        _, sv, Vt = mpmath.svd_r(Mm, compute_uv=True)
        order_idx = sorted(range(k), key=lambda r: -sv[r])
        V = [from_fraction(n, _mpf_fraction(mpmath.mpf(Vt[order_idx[r], i])))
             for r in range(k) for i in range(k)]  # column r of V, row i
        sig = [from_fraction(n, _mpf_fraction(mpmath.mpf(sv[order_idx[r]]))) for r in range(k)]
    lam = sig
    root = [mp_sqrt(n, v) for v in lam]
    lis = [mp_recip(n, v) for v in root]
    R = [mp_mul(n, exact_dot(n, [(L1[i + q * k], V[q + r * k]) for q in range(i + 1)]), lis[r])
         for r in range(k) for i in range(k)]
    X = [Mp(n)] * (k * k)  # L1' X = V by back substitution (xtrsm_lower, transposed)
    for r in range(k):
        for i in range(k - 1, -1, -1):
            d = mp_sub(n, V[i + r * k], exact_dot(n, [(L1[q + i * k], X[q + r * k]) for q in range(i + 1, k)]))
            X[i + r * k] = mp_div(n, d, L1[i + i * k])
    Rinv = [mp_mul(n, X[j + r * k], root[r]) for j in range(k) for r in range(k)]
    G = [exact_dot(n, [(R[i + q * k], R[j + q * k]) for q in range(k)]) if i <= j else Mp(n)
         for j in range(k) for i in range(k)]
    return lam, lis, R, Rinv, G


# ------------------------------------------------------------------------------------------
# Step-length bound of one PSD block at MPFR width (psdtrianglecone.rs:1041-1072
# step_component_inner, 1180-1231 step_length_psd_component, 1233-1285 eigval_min_f64,
# 1287-1390 min_eigenvalue_f64, 1168-1178 admits, 1391-1406 lrscale_symmetric).
# ------------------------------------------------------------------------------------------
def mp_add(n: int, a: Mp, b: Mp) -> Mp:
    return from_fraction(n, a.fraction() + b.fraction())


def min_eigenvalue_f64(a: List[float], n: int):
    """The reference's binary64 Householder tridiagonalisation and Sturm bisection, in its
    operation order (Python floats round each operation, as Rust does)."""
    a = list(a)

    def at(i, j):
        return i + j * n
    d = [0.0] * n
    e = [0.0] * n
    for i in range(n - 1, 0, -1):
        l = i - 1
        h = 0.0
        if l > 0:
            scale = -0.0
            for k in range(l + 1):
                scale += abs(a[at(i, k)])
            if scale == 0.0:
                e[i] = a[at(i, l)]
            else:
                for k in range(l + 1):
                    a[at(i, k)] /= scale
                    h += a[at(i, k)] * a[at(i, k)]
                f = a[at(i, l)]
                g = -math.sqrt(h) if f >= 0.0 else math.sqrt(h)
                e[i] = scale * g
                h -= f * g
                a[at(i, l)] = f - g
                f = 0.0
                for j in range(l + 1):
                    g = 0.0
                    for k in range(j + 1):
                        g += a[at(j, k)] * a[at(i, k)]
                    for k in range(j + 1, l + 1):
                        g += a[at(k, j)] * a[at(i, k)]
                    e[j] = g / h
                    f += e[j] * a[at(i, j)]
                hh = f / (h + h)
                for j in range(l + 1):
                    f = a[at(i, j)]
                    g = e[j] - hh * f
                    e[j] = g
                    for k in range(j + 1):
                        a[at(j, k)] -= f * e[k] + g * a[at(i, k)]
        else:
            e[i] = a[at(i, l)]
        d[i] = h
    e[0] = 0.0
    for i in range(n):
        d[i] = a[at(i, i)]
    eps = 2.0 ** -52
    tiny = 2.0 ** -1022 / eps

    def below(x):
        count = 0
        q = d[0] - x
        for i in range(n):
            if i > 0:
                q = d[i] - x - e[i] * e[i] / q
            if q == 0.0:
                q = -tiny
            if q < 0.0:
                count += 1
        return count
    lo, hi = math.inf, -math.inf
    for i in range(n):
        r = abs(e[i]) + (abs(e[i + 1]) if i + 1 < n else 0.0)
        lo = min(lo, d[i] - r)
        hi = max(hi, d[i] + r)
    if not (math.isfinite(lo) and math.isfinite(hi)):
        return None
    width = max(hi - lo, max(abs(hi), abs(lo)) * eps)
    lo -= width * eps
    hi += width * eps
    for _ in range(128):
        mid = 0.5 * (lo + hi)
        if mid <= lo or mid >= hi:
            break
        if below(mid) >= 1:
            hi = mid
        else:
            lo = mid
    return 0.5 * (lo + hi)


def step_component(n: int, k: int, d: List[Mp], Rx: List[Mp], lis: List[Mp], primal: bool, amax: Mp):
    """Returns (alpha, path): path 0 a priori binary64 bound, 1 certified by the exact Cholesky of
    I + alpha_c Delta, 2 the full-precision eigensolver (here mpmath at 64 extra bits)."""
    import mpmath
    f = frac_1_sqrt2(n)
    Xm = [Mp(n)] * (k * k)
    for c in range(k):
        for r in range(k):
            lo, hi = min(r, c), max(r, c)
            v = d[hi * (hi + 1) // 2 + lo]
            Xm[r + c * k] = v if r == c else mp_mul(n, v, f)
    Y = congruence(n, "N" if primal else "T", k, k, Rx, k, Xm, k)
    D = [Mp(n)] * (k * k)
    for c in range(k):
        for r in range(c + 1):
            v = Y[r + c * k]
            if r != c:
                two = v if v.is_zero() else Mp(n, v.neg, v.mant, v.exp + 1)
                v = mp_mul(n, mp_mul(n, two, f), f)
            v = mp_mul(n, v, mp_mul(n, lis[r], lis[c]))
            D[r + c * k] = D[c + r * k] = v

    def finish(gamma: Mp, path: int):
        if not gamma.is_zero() and gamma.neg:
            a = mp_recip(n, gamma)
            a = Mp(n, not a.neg, a.mant, a.exp)
            return (a if a.fraction() < amax.fraction() else amax), path
        return amax, path
    if k > 3:
        amx = float(amax.fraction())
        vals = [float(v.fraction()) for v in D]
        if all(math.isfinite(v) and abs(v) <= 1e150 for v in vals) and math.isfinite(amx):
            sumsq = 0.0
            for v in vals:
                sumsq += v * v
            gamma = min_eigenvalue_f64(vals, k)
            if gamma is not None:
                bound = 2.0 * float((k + 1) ** 2) * 2.0 ** -52 * math.sqrt(sumsq)
                floor = 1.0 / amx if (amx > 0.0 and math.isfinite(amx)) else 0.0
                if bound <= 1e-10 * max(abs(gamma), floor):
                    return finish(mp_from_float(n, gamma), 0)
                alc = mp_from_float(n, -(1.0 - 1e-10) / gamma) if (gamma < 0.0 and -1.0 / gamma < amx) else amax
                C = [mp_mul(n, v, alc) for v in D]
                for i in range(k):
                    C[i + i * k] = mp_add(n, C[i + i * k], mp_one(n))
                if xpotrf(n, "L", k, C, k) == 0:
                    return finish(mp_from_float(n, gamma), 1)
    with mpmath.workprec(64 * n + 64):
        Mm = mpmath.matrix(k, k)
        for c in range(k):
            for r in range(k):
                fr = D[r + c * k].fraction()
                Mm[r, c] = mpmath.mpf(fr.numerator) / fr.denominator
        ev = mpmath.eigsy(Mm, eigvals_only=True)
        lam = min(ev[i] for i in range(k))
        return finish(from_fraction(n, _mpf_fraction(lam)), 2)
