"""Rank-one (Gram) form of the PSD constraint operator against the ordinary dense-column form.

A PSD block whose every constraint column is rank one (sigma u u') is stored as its factor and
its Schur block, forward and adjoint products are computed from V = Rinv U (the algebra of the
reference's sampled Gram update, sampled/mod.rs:1973-2025).  Bars:
  * detection: rank-one blocks of the bootstrap generator are all Gram, dense SDP blocks none;
  * operators: A x and A' z within 1e-13 relative of scipy on the CSC input;
  * Schur block: within 1e-11 relative of the oracle (test_gpu_parity covers the same fixture);
  * whole solves: Gram and ordinary forms (SDPX_B200_GRAM=0) and the oracle agree in status,
    iterations within 1 and objective within 1e-8 relative, also on a problem mixing both forms.
"""
import os

import numpy as np
import pytest
import scipy.sparse as sp

from oracle import ipm
from sdpx_b200 import problems as P
from sdpx_b200.solver import DefaultSettings, DefaultSolver, KernelContext

pytestmark = pytest.mark.gpu


def _solver(prob, gram=True):
    old = os.environ.get("SDPX_B200_GRAM")
    os.environ["SDPX_B200_GRAM"] = "1" if gram else "0"
    try:
        return DefaultSolver(prob.P, prob.q, prob.A, prob.b, prob.cones,
                             DefaultSettings(kkt_form="condensed"))
    finally:
        if old is None:
            del os.environ["SDPX_B200_GRAM"]
        else:
            os.environ["SDPX_B200_GRAM"] = old


def _mixed_problem(seed=2):
    """Rank-one bootstrap blocks plus one dense PSD block on the same constraints (X0 = I)."""
    base = P.rank1_sdp(4, 60, seed=seed, nmin=5, nmax=12)
    rng = np.random.default_rng(seed + 100)
    nd, m = 6, base.n
    cols, trs = [], []
    for _ in range(m):
        B = rng.standard_normal((nd, nd))
        Ai = (B + B.T) / 2
        cols.append(P.svec(Ai))
        trs.append(np.trace(Ai))
    Ad = np.array(cols).T
    y0 = base.meta["y0"]
    Cd = P.smat(Ad @ y0, nd) + np.eye(nd)
    A = sp.vstack([base.A, sp.csc_matrix(Ad)]).tocsc()
    return P.ConicProblem(P=None, q=base.q - np.array(trs), A=A,
                          b=np.concatenate([base.b, P.svec(Cd)]),
                          cones=base.cones + [("psd", nd)], rank1=None, name="mixed", meta={})


def test_detection_counts():
    r1 = _solver(P.rank1_sdp(8, 200, seed=1, nmin=6, nmax=24))
    assert r1.schur_forms() == {"gram": 8, "ordinary": 0}
    dense = _solver(P.dense_sdp(12, 40, seed=0))
    assert dense.schur_forms() == {"gram": 0, "ordinary": 1}
    mixed = _solver(_mixed_problem())
    assert mixed.schur_forms() == {"gram": 4, "ordinary": 1}
    off = _solver(P.rank1_sdp(8, 200, seed=1, nmin=6, nmax=24), gram=False)
    assert off.schur_forms() == {"gram": 0, "ordinary": 8}


@pytest.mark.parametrize("gram", [True, False])
def test_operator_products_match_csc(gram):
    prob = _mixed_problem(seed=5)
    old = os.environ.get("SDPX_B200_GRAM")
    os.environ["SDPX_B200_GRAM"] = "1" if gram else "0"
    try:
        ctx = KernelContext()
        ctx.upload(prob.A, [d for _, d in prob.cones])
    finally:
        if old is None:
            del os.environ["SDPX_B200_GRAM"]
        else:
            os.environ["SDPX_B200_GRAM"] = old
    ctx.identity_scaling()
    g = np.random.default_rng(3)
    x, z = g.standard_normal(prob.n), g.standard_normal(prob.m)
    A = sp.csc_matrix(prob.A)
    zn, zm = np.zeros(prob.n), np.zeros(prob.m)
    _, ez, _ = ctx.residual(zn, zm, x, zm)  # ez = -A x
    ex, _, _ = ctx.residual(zn, zm, zn, z)  # ex = -A' z
    ax, atz = A @ x, A.T @ z
    assert np.max(np.abs(-ez - ax)) <= 1e-13 * np.max(np.abs(A).sum(axis=1)) * np.max(np.abs(x))
    assert np.max(np.abs(-ex - atz)) <= 1e-13 * np.max(np.abs(A).sum(axis=0)) * np.max(np.abs(z))


def test_gram_schur_matches_ordinary():
    prob = _mixed_problem(seed=7)
    s, z = [], []
    rng = np.random.default_rng(1)
    for _, d in prob.cones:
        for out in (s, z):
            B = rng.standard_normal((d, d))
            out.append(P.svec(B @ B.T / d + 0.1 * np.eye(d)))
    s, z = np.concatenate(s), np.concatenate(z)
    H = {}
    for gram in (True, False):
        old = os.environ.get("SDPX_B200_GRAM")
        os.environ["SDPX_B200_GRAM"] = "1" if gram else "0"
        try:
            ctx = KernelContext()
            ctx.upload(prob.A, [d for _, d in prob.cones])
        finally:
            if old is None:
                del os.environ["SDPX_B200_GRAM"]
            else:
                os.environ["SDPX_B200_GRAM"] = old
        assert ctx.nt_scale(s, z)[1] == 0
        H[gram] = ctx.schur()
    assert np.array_equal(H[True], H[True].T)
    assert np.max(np.abs(H[True] - H[False])) <= 1e-12 * np.max(np.abs(H[False]))
    # both against the oracle's Schur complement (per PSD block, condensed/psd.rs:1299-1570)
    A = sp.csc_matrix(prob.A)
    Ho = np.zeros((prob.n, prob.n))
    r0 = 0
    for _, d in prob.cones:
        t = d * (d + 1) // 2
        cone = ipm.PsdCone(d)
        assert cone.update_scaling(s[r0:r0 + t], z[r0:r0 + t])
        sub = A[r0:r0 + t, :]
        cols = np.flatnonzero(sub.getnnz(axis=0))
        Ho[np.ix_(cols, cols)] += cone.schur_block(sub[:, cols].toarray())
        r0 += t
    for form in (True, False):
        assert np.max(np.abs(H[form] - Ho)) <= 1e-11 * np.max(np.abs(Ho))


@pytest.mark.parametrize("maker", [lambda: P.rank1_sdp(8, 200, seed=1, nmin=6, nmax=24),
                                   lambda: _mixed_problem(seed=3)])
def test_whole_solve_gram_vs_ordinary_vs_oracle(maker):
    prob = maker()
    o = ipm.solve(prob)
    res = {}
    for gram in (True, False):
        s = _solver(prob, gram)
        s.solve()
        res[gram] = s.solution
        assert s.solution.status_code == o.status, (gram, s.solution.status, o.status)
        assert abs(s.solution.iterations - o.iterations) <= 1
        assert abs(s.solution.obj_val - o.objective) <= 1e-8 * max(1.0, abs(o.objective))
    assert abs(res[True].iterations - res[False].iterations) <= 1
