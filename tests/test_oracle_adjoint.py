"""The oracle's adjoint (oracle/adjoint.py) against central finite differences of oracle solves.

The reference has no adjoint, so this is the oracle's own pin: on a small conic QP (orthant rows
and one PSD block) solved to gap 1e-10, the directional derivative of L = 1/2 |x* - t|^2 along
random directions in (q, b, A) matches central differences with h = 1e-5 to 1e-3 relative.
"""
import numpy as np
import scipy.sparse as sp

from oracle import adjoint as oracle_adjoint
from oracle import ipm
from sdpx_b200 import problems as P

TOL = dict(tol_gap_abs=1e-10, tol_gap_rel=1e-10, tol_feas=1e-10)


def _solve(prob, **kw):
    q = P.ConicProblem(P=prob.P, q=kw.get("q", prob.q), A=kw.get("A", prob.A), b=kw.get("b", prob.b),
                       cones=prob.cones, rank1=None, name=prob.name, meta=prob.meta)
    r = ipm.solve(q, **TOL)
    assert r.status in (ipm.SOLVED, ipm.ALMOST_SOLVED), r.status
    return r


def test_oracle_adjoint_matches_finite_differences():
    prob = P.conic_qp(1, n=12, n_nn=8, psd=3, rank=4)
    t = prob.meta["t"]
    r = _solve(prob)
    dq, db, dA = oracle_adjoint.adjoint(prob, r.x, r.s, r.z, r.x - t)
    A = sp.csc_matrix(prob.A)
    rng = np.random.default_rng(3)
    h = 1e-5
    for _ in range(2):
        vq = rng.standard_normal(prob.n)
        vb = rng.standard_normal(prob.m)
        vA = sp.csc_matrix((rng.standard_normal(A.nnz), A.indices, A.indptr), shape=A.shape)
        analytic = dq @ vq + db @ vb + float(dA.multiply(vA).sum())
        xp = _solve(prob, q=prob.q + h * vq, b=prob.b + h * vb, A=A + h * vA).x
        xm = _solve(prob, q=prob.q - h * vq, b=prob.b - h * vb, A=A - h * vA).x
        fd = (0.5 * np.sum((xp - t) ** 2) - 0.5 * np.sum((xm - t) ** 2)) / (2 * h)
        assert abs(analytic - fd) <= 1e-3 * max(1.0, abs(fd)), (analytic, fd)
