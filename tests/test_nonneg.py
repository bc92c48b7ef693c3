"""Nonnegative-orthant cones on the GPU path (conic QPs of the differentiation workload).

Bars (as the other whole-solve parity tests): same status as the oracle, iterations within 1,
objective within 1e-8 relative, primal solution within 1e-6; an orthant-only LP and mixed
orthant + PSD problems with a quadratic objective, the orthant before or after the PSD block.
"""
import numpy as np
import pytest
import scipy.sparse as sp

from oracle import ipm
from sdpx_b200 import problems as P
from sdpx_b200.solver import DefaultSettings, solve_problem

pytestmark = pytest.mark.gpu


def _parity(prob):
    o = ipm.solve(prob)
    g = solve_problem(prob, DefaultSettings(kkt_form="condensed")).solution
    assert g.status_code == o.status, (g.status, o.status)
    assert abs(g.iterations - o.iterations) <= 1, (g.iterations, o.iterations)
    assert abs(g.obj_val - o.objective) <= 1e-8 * max(1.0, abs(o.objective))
    assert np.max(np.abs(g.x - o.x)) <= 1e-6 * max(1.0, np.max(np.abs(o.x)))
    return g, o


@pytest.mark.parametrize("kw", [dict(n=20, n_nn=15, psd=4, rank=5), dict(n=60, n_nn=40, psd=8, rank=10),
                                dict()])
def test_conic_qp_parity(kw):
    _parity(P.conic_qp(3, **kw))


def test_orthant_after_psd_block():
    p = P.conic_qp(5, n=30, n_nn=12, psd=5, rank=6)
    k = 12
    A = sp.vstack([p.A[k:], p.A[:k]]).tocsc()  # PSD rows first, then the orthant
    b = np.concatenate([p.b[k:], p.b[:k]])
    q = P.ConicProblem(P=p.P, q=p.q, A=A, b=b, cones=[("psd", 5), ("nonneg", 12)], rank1=None,
                       name="qp_psd_first", meta={})
    _parity(q)


def test_orthant_only_lp():
    rng = np.random.default_rng(2)
    n, m = 15, 40
    A = rng.standard_normal((m, n))
    x0 = rng.standard_normal(n)
    b = A @ x0 + 1.0
    c = -A.T @ rng.uniform(0.5, 1.5, m)  # dual feasible: A'z + c = 0 with z > 0
    p = P.ConicProblem(P=None, q=c, A=sp.csc_matrix(A), b=b, cones=[("nonneg", m)], rank1=None,
                       name="lp", meta={})
    _parity(p)
