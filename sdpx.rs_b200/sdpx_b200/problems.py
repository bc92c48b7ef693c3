"""Conic problem container and the synthetic SDP generators.

The conic form is the one SDPX solves (crates/solver/src/solver/default/solver.rs:260,
include/sdpx.h:19-46):

    minimize    1/2 x'Px + q'x
    subject to  b - A x = s,  s in K

with K a product of cones.  PSD cones use the reference's triangle convention: the upper
triangle in column order with off-diagonal entries scaled by sqrt(2)
(include/sdpx.h:32-33).

The generators restate the synthetic workloads used to measure the hot path:

* ``dense_sdp``   one PSD block n=50, m=200 dense symmetric constraints (the CPU-runnable case);
* ``rank1_sdp``   many PSD blocks with Chebyshev bases, each constraint a sum of four rank-one
                  terms ``w v v'`` (a bootstrap-shaped SDP);
* ``batch_sdps``  independent small dense SDPs drawn from seed + index.

Every SDP is posed in dual form: x = y, P = 0, q = -b_primal, column i of A = svec(A_i) over
the stacked PSD blocks, conic b = svec(C).  With X0 = I primal feasible and C = sum y0_i A_i + I
the problem is strictly primal and dual feasible.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Optional, Tuple

import numpy as np
import scipy.sparse as sp

SQRT2 = float(np.sqrt(2.0))


def tri(n: int) -> int:
    return n * (n + 1) // 2


def svec_index(n: int) -> Tuple[np.ndarray, np.ndarray]:
    """(row, col) of each svec slot: upper triangle, column order."""
    j, i = np.tril_indices(n)  # tril row-major == upper column-major, transposed
    return i, j


def svec(M: np.ndarray) -> np.ndarray:
    n = M.shape[0]
    i, j = svec_index(n)
    v = M[i, j].astype(np.float64, copy=True)
    v[i != j] *= SQRT2
    return v


def smat(v: np.ndarray, n: int) -> np.ndarray:
    i, j = svec_index(n)
    M = np.zeros((n, n))
    w = np.where(i == j, v, v / SQRT2)
    M[i, j] = w
    M[j, i] = w
    return M


@dataclass
class Rank1Terms:
    """Rank-one (Gram) description of a PSD constraint operator.

    Constraint ``i`` restricted to block ``j`` is ``sum w v v'`` over the terms (i, j, c, w),
    ``v = bases[j][:, c]``.  This is algebraically the CSC operator ``A``; a solver may use
    either description.  ``terms`` rows are (constraint, block, column) int64, ``weights``
    float64, sorted by constraint then block.
    """
    bases: List[np.ndarray]
    terms: np.ndarray
    weights: np.ndarray


@dataclass
class ConicProblem:
    P: Optional[sp.csc_matrix]
    q: np.ndarray
    A: sp.csc_matrix
    b: np.ndarray
    cones: List[Tuple[str, int]]
    rank1: Optional[Rank1Terms] = None
    name: str = ""
    meta: dict = field(default_factory=dict)

    @property
    def n(self) -> int:
        return int(self.A.shape[1])

    @property
    def m(self) -> int:
        return int(self.A.shape[0])

    def cone_rows(self) -> List[Tuple[str, int, int, int]]:
        """(kind, dim, row_start, row_count) per cone."""
        out, r = [], 0
        for kind, d in self.cones:
            cnt = tri(d) if kind == "psd" else d
            out.append((kind, d, r, cnt))
            r += cnt
        return out


def _chebyshev_basis(n: int, s: int) -> np.ndarray:
    x = np.cos((2 * np.arange(s) + 1) * np.pi / (2 * s))
    V = np.empty((n, s))
    V[0] = 1.0
    if n > 1:
        V[1] = x
    for r in range(2, n):
        V[r] = 2 * x * V[r - 1] - V[r - 2]
    return V


def dense_sdp(n: int = 50, m: int = 200, seed: int = 0) -> ConicProblem:
    """One PSD block of order n and m dense symmetric constraints.

    A_i: upper entries (diagonal included) iid N(0,1); X0 = I; b_i = tr(A_i);
    y0 ~ N(0,1)^m; C = sum_i y0_i A_i + I.
    """
    rng = np.random.default_rng(seed)
    t = tri(n)
    i, j = svec_index(n)
    U = rng.standard_normal((m, t))  # upper entries, column order
    y0 = rng.standard_normal(m)
    cols = U.copy()
    cols[:, i != j] *= SQRT2  # svec(A_i)
    bprim = U[:, i == j].sum(axis=1)  # tr(A_i X0) with X0 = I
    Csvec = y0 @ cols + svec(np.eye(n))
    A = sp.csc_matrix(cols.T)
    return ConicProblem(P=None, q=-bprim, A=A, b=Csvec, cones=[("psd", n)],
                        name=f"dense_sdp_n{n}_m{m}_s{seed}",
                        meta={"seed": seed, "y0": y0})


def rank1_sdp(blocks: int = 32, m: int = 2000, seed: int = 0, nmin: int = 10, nmax: int = 60,
              touch: int = 4) -> ConicProblem:
    """Bootstrap-shaped SDP: ``blocks`` PSD blocks with Chebyshev bases V_j (n_j x 2n_j).

    Each constraint touches ``touch`` distinct blocks; in each a basis column c ~ U{0..s_j-1}
    and weight w ~ U[0.5, 2] give the term w v v'.  X0 = I, b_i = sum w |v|^2, y0 ~ N(0,1),
    C_j = sum_i y0_i A_ij + I.
    """
    rng = np.random.default_rng(seed)
    ns = rng.integers(nmin, nmax + 1, size=blocks)
    bases = [_chebyshev_basis(int(nj), 2 * int(nj)) for nj in ns]
    terms = np.empty((m * touch, 3), dtype=np.int64)
    weights = np.empty(m * touch)
    k = 0
    for c_i in range(m):
        bl = np.sort(rng.choice(blocks, size=touch, replace=False))
        for j in bl:
            s_j = bases[j].shape[1]
            col = int(rng.integers(0, s_j))
            w = float(rng.uniform(0.5, 2.0))
            terms[k] = (c_i, j, col)
            weights[k] = w
            k += 1
    y0 = rng.standard_normal(m)
    bprim = np.zeros(m)
    sq = [np.sum(V * V, axis=0) for V in bases]
    for (ci, j, col), w in zip(terms, weights):
        bprim[ci] += w * sq[j][col]
    # C_j = V_j diag(sum of y0_i w over terms on column c) V_j' + I
    offs = np.concatenate([[0], np.cumsum([tri(int(nj)) for nj in ns])])
    bcon = np.zeros(offs[-1])
    for j, V in enumerate(bases):
        sel = terms[:, 1] == j
        d = np.zeros(V.shape[1])
        np.add.at(d, terms[sel, 2], y0[terms[sel, 0]] * weights[sel])
        C = (V * d) @ V.T + np.eye(V.shape[0])
        bcon[offs[j]:offs[j + 1]] = svec(C)
    # CSC operator: column i stacks svec(w v v') on the rows of its blocks
    rows, vals, colidx = [], [], []
    for (ci, j, col), w in zip(terms, weights):
        v = bases[j][:, col]
        sv = svec(w * np.outer(v, v))
        rows.append(offs[j] + np.arange(sv.size))
        vals.append(sv)
        colidx.append(np.full(sv.size, ci))
    A = sp.csc_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(colidx))),
                      shape=(offs[-1], m))
    A.sort_indices()
    return ConicProblem(P=None, q=-bprim, A=A, b=bcon,
                        cones=[("psd", int(nj)) for nj in ns],
                        rank1=Rank1Terms(bases=bases, terms=terms, weights=weights),
                        name=f"rank1_sdp_b{blocks}_m{m}_s{seed}",
                        meta={"seed": seed, "y0": y0})


def batch_sdps(count: int, seed: int = 0, nrange=(8, 64), mrange=(20, 300)) -> List[ConicProblem]:
    """Independent small dense SDPs, instance b drawn from seed + b."""
    out = []
    for b in range(count):
        rng = np.random.default_rng(seed + b)
        n = int(rng.integers(nrange[0], nrange[1] + 1))
        m = int(rng.integers(mrange[0], mrange[1] + 1))
        out.append(dense_sdp(n, m, seed=(seed + b) * 7919 + 1))
    return out


def conic_qp(seed: int = 0, n: int = 200, n_nn: int = 150, psd: int = 20, rank: int = 50) -> ConicProblem:
    """Conic QP of the differentiation workload: min 1/2 x'Px + q'x s.t. b - Ax in K.

    x in R^n; P = L L' + 0.1 I with L (n x rank) iid N(0, 1/rank); q ~ N(0, 1); K = the
    nonnegative orthant of dimension n_nn followed by one PSD triangle cone of order psd;
    A (n_nn + tri(psd) x n) iid N(0, 1/sqrt(n)); x0 ~ N(0, 1); s0 strictly interior (orthant
    entries 1, PSD part svec(I)); b = A x0 + s0.  The second argument of N(., .) is the
    variance for both L and A.  A loss target t ~ N(0, 1)^n is stored in meta["t"].
    """
    rng = np.random.default_rng(seed)
    L = rng.standard_normal((n, rank)) * np.sqrt(1.0 / rank)
    Pm = L @ L.T + 0.1 * np.eye(n)
    q = rng.standard_normal(n)
    rows = n_nn + tri(psd)
    A = rng.standard_normal((rows, n)) * np.sqrt(1.0 / np.sqrt(n))
    x0 = rng.standard_normal(n)
    s0 = np.concatenate([np.ones(n_nn), svec(np.eye(psd))])
    b = A @ x0 + s0
    t = rng.standard_normal(n)
    return ConicProblem(P=sp.csc_matrix(Pm), q=q, A=sp.csc_matrix(A), b=b,
                        cones=[("nonneg", n_nn), ("psd", psd)],
                        name=f"conic_qp_n{n}_nn{n_nn}_psd{psd}_s{seed}",
                        meta={"seed": seed, "t": t, "x0": x0})


def basic_projection_sdp() -> ConicProblem:
    """Known-answer projection problem: min 1/2|x|^2 s.t. b - x in PSD(3).

    Data of crates/solver/tests/it/basic_sdp.rs:5-25 (P = I, A = I, q = 0).
    """
    P = sp.identity(6, format="csc")
    A = sp.identity(6, format="csc")
    return ConicProblem(P=P, q=np.zeros(6), A=A, b=np.array([-3., 1., 4., 1., 2., 5.]),
                        cones=[("psd", 3)], name="basic_projection_sdp")


def sampled_two_by_two(scale: float = 1.0) -> ConicProblem:
    """Known-answer sampled SDP of crates/solver/tests/it/sampled_solver.rs:8-25.

    One PSD block of order 2, basis columns (1, 1/4) and (1/4, 1), weights -1:
    minimize x0 + x1 s.t. -I*scale + x0 v0 v0' + x1 v1 v1' >= 0.  Answer x = 16/9 * scale.
    """
    V = np.array([[1.0, 0.25], [0.25, 1.0]])
    cols = [svec(-np.outer(V[:, k], V[:, k])) for k in range(2)]
    A = sp.csc_matrix(np.stack(cols, axis=1))
    b = np.array([-1.0, 0.0, -1.0]) * scale
    r1 = Rank1Terms(bases=[V], terms=np.array([[0, 0, 0], [1, 0, 1]], dtype=np.int64),
                    weights=np.array([-1.0, -1.0]))
    return ConicProblem(P=None, q=np.ones(2), A=A, b=b, cones=[("psd", 2)], rank1=r1,
                        name="sampled_two_by_two")
